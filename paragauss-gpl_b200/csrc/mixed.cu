// mixed.cu -- mixed-precision XC build on the fifth-generation tensor cores.
//
// Both dense contractions run on tcgen05 kind::i8 with exact 32-bit integer
// accumulation, using an Ozaki-type split of the operands:
//   every row (or column) of an operand is scaled by a power of two so its
//   largest entry lies in [1/2, 1), rounded to a 34-bit fixed-point integer
//   and written as 5 balanced base-128 digits (signed 8-bit, |digit| <= 64).
//   The product of two operands is the sum over digit pairs (s, t) weighted
//   by 2^(-12-7(s+t)); pairs with s + t <= 4 are kept (15 MMAs per K step),
//   grouped by s + t into 5 TMEM accumulators, and recombined in FP64.
// Integer accumulation is exact, so the only errors are the 34-bit operand
// rounding and the dropped pairs (about 2^-35 of the row scale).  Split-BF16
// products accumulated in FP32 were measured against the FP64 oracle and
// rejected: the tensor core's FP32 accumulation gives a systematic bias that
// grows with K (|dE_xc| = 5.5e-3 Eh on the 60-atom workload).
//
// Precision plan of the mode (every choice measured against the oracle):
//   * basis values and gradients evaluated and stored in FP64; FP32 storage
//     of phi / grad phi / Z limited |dE_xc| to ~6e-6 and |dV_xc| to ~1e-5 on
//     the 60-atom workload;
//   * X = phi^T P (density-matrix form) on the integer tensor cores, then
//     rho = sum X phi and grad rho = 2 sum X grad phi in FP64 per point;
//   * functional in FP64, E_xc and N_el in FP64 with Kahan compensation;
//   * ham = Z^T phi on the integer tensor cores, FP64 partial tiles.
//
// Kernels: basis (k_basis_l, shared with the FP64 path), k_oz_quant_* (scales and
// operand tiles),
// k_oz_density (tcgen05), k_oz_zbuild, k_oz_vpot (tcgen05), k_oz_pack.
// Tiles are 128 x 96: five 96-column INT32 accumulators fill 480 of the 512
// TMEM columns.
#include <cstdint>
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>

#include "kernels.h"
#include "mixed.h"
#include "ozaki.cuh"
#include "tc.cuh"

namespace pgxc {

namespace {

constexpr int kRowsA = 128;          // M of every MMA
constexpr int kRowsB = 96;           // N of every MMA
constexpr int kBlkA = kRowsA * 32;   // one slice of a 128-row x 32-byte K block
constexpr int kBlkB = kRowsB * 32;
constexpr int kOpA = kSlices * kBlkA;
constexpr int kOpB = kSlices * kBlkB;
constexpr int kStages = 5;           // bulk-copy ring depth
constexpr int kKStep = 32;           // K elements per int8 MMA
constexpr int kAlignFn = 384;        // functions padded to lcm(128, 96)

}  // namespace

struct MixedState {
  int64_t nbas = 0, ldk = 0, ldp = 0;
  bool gga = false;
  double *phi = nullptr, *gx = nullptr, *gy = nullptr, *gz = nullptr, *Z = nullptr;  // [ldk][ldp]
  double* P = nullptr;          // [ldk][ldk]
  int8_t* tA1 = nullptr;        // density A: phi, per-point scales      [pb][ks][slice][128 x 32]
  int8_t* tB1 = nullptr;        // density B: P, per-row scales          [nb][ks][slice][96 x 32]
  int8_t* tZ = nullptr;         // potential A: Z, per-function scales   [fb][ks][slice][128 x 32]
  int8_t* tP2 = nullptr;        // potential B: phi, per-function scales [gb][ks][slice][96 x 32]
  int* e_pt = nullptr;          // [ldp]
  int* e_P = nullptr;           // [ldk]
  int* e_Z = nullptr;           // [ldk]
  int* e_fn = nullptr;          // [ldk]
  unsigned long long* zmax = nullptr;   // [ldk] bit patterns of max |Z|
  unsigned long long* fmax = nullptr;   // [ldk] bit patterns of max |phi|
  int nta = 0, ntb = 0, ntiles = 0, nsplit = 0, ks_per_split = 0;
  int* err = nullptr;
  double* vpart = nullptr;
  std::vector<void*> allocs;
};

namespace {

template <typename T>
cudaError_t mx_alloc(MixedState* m, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) {
    m->allocs.push_back(q);
    *p = (T*)q;
  }
  return e;
}

__global__ void k_oz_fexp(const unsigned long long* __restrict__ mx, int64_t n, int* __restrict__ e) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) e[i] = scale_exp(__longlong_as_double((long long)mx[i]));
}

// per row of the symmetric density matrix (= per column)
__global__ void k_oz_rowexp_P(const double* __restrict__ P, int64_t ldk, int* __restrict__ e) {
  const double* row = P + (int64_t)blockIdx.x * ldk;
  double mx = 0.0;
  for (int64_t j = threadIdx.x; j < ldk; j += blockDim.x) mx = fmax(mx, fabs(row[j]));
  __shared__ double red[256];
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) e[blockIdx.x] = scale_exp(red[0]);
}

// ---------------------------------------------------------------------------
// operand tiles: block (rb, kb) = ROWS rows from rb*ROWS, K from kb*32 ->
// [rb][kb][slice][ROWS x 32]; thread t owns row t and writes one 16-byte
// core-matrix row per (slice, K half).
// ---------------------------------------------------------------------------
template <int ROWS>
__device__ __forceinline__ void store_row(int8_t* dst, int t, int h, const int8_t (&d)[kSlices][16]) {
#pragma unroll
  for (int s = 0; s < kSlices; ++s)
    *reinterpret_cast<uint4*>(dst + s * (ROWS * 32) + blk_off(t, h * 16)) = *reinterpret_cast<const uint4*>(d[s]);
}

// rows = points, K = functions: element (p, f) = phi[f][p].  One block per
// 128 points: the per-point scale (largest |phi| over all functions) is found
// first, then every K block of the 128 rows is quantized.
__global__ void __launch_bounds__(128) k_oz_quant_pts(const double* __restrict__ phi, int64_t ldp, int64_t nbas,
                                                      int nks, int* __restrict__ e_pt, int8_t* __restrict__ out) {
  const int pb = blockIdx.x, t = threadIdx.x;
  const int64_t p = (int64_t)pb * 128 + t;
  double m8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t f = 0;
  for (; f + 8 <= nbas; f += 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j) m8[j] = fmax(m8[j], fabs(phi[(f + j) * ldp + p]));
  }
  for (; f < nbas; ++f) m8[0] = fmax(m8[0], fabs(phi[f * ldp + p]));
  double mx = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) mx = fmax(mx, m8[j]);
  const int e = scale_exp(mx);
  e_pt[p] = e;
  for (int kb = 0; kb < nks; ++kb) {
    int8_t* dst = out + ((int64_t)pb * nks + kb) * kOpA;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      alignas(16) int8_t d[kSlices][16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        int8_t q[kSlices];
        digits(phi[(int64_t)(kb * 32 + h * 16 + k) * ldp + p], e, q);
#pragma unroll
        for (int s = 0; s < kSlices; ++s) d[s][k] = q[s];
      }
      store_row<128>(dst, t, h, d);
    }
  }
}

// rows = functions (blocks of ROWS), K = points: element (f, p) = a[f][p], per-function scale
template <int ROWS>
__global__ void __launch_bounds__(kBlock4(ROWS)) k_oz_quant_fn(const double* __restrict__ a, int64_t ldp,
                                                               const int* __restrict__ e_fn, int nks,
                                                               int8_t* __restrict__ out) {
  const int fb = blockIdx.x, kb = blockIdx.y, t = threadIdx.x;
  if (t >= ROWS) return;
  const int64_t f = (int64_t)fb * ROWS + t;
  const int e = e_fn[f];
  const double2* src = reinterpret_cast<const double2*>(a + f * ldp + (int64_t)kb * 32);
  int8_t* dst = out + ((int64_t)fb * nks + kb) * (kSlices * ROWS * 32);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    alignas(16) int8_t d[kSlices][16];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const double2 x = __ldg(src + h * 8 + v);
      int8_t q0[kSlices], q1[kSlices];
      digits(x.x, e, q0);
      digits(x.y, e, q1);
#pragma unroll
      for (int s = 0; s < kSlices; ++s) {
        d[s][2 * v] = q0[s];
        d[s][2 * v + 1] = q1[s];
      }
    }
    store_row<ROWS>(dst, t, h, d);
  }
}

// density B: rows = nu (blocks of 96), K = mu, element P[mu][nu] = P[nu][mu], per-row scale
__global__ void __launch_bounds__(kBlock4(kRowsB)) k_oz_quant_P(const double* __restrict__ P, int64_t ldk,
                                                                const int* __restrict__ e_P, int nks,
                                                                int8_t* __restrict__ out) {
  const int nb = blockIdx.x, kb = blockIdx.y, t = threadIdx.x;
  if (t >= kRowsB) return;
  const int64_t nu = (int64_t)nb * kRowsB + t;
  const int e = e_P[nu];
  int8_t* dst = out + ((int64_t)nb * nks + kb) * kOpB;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    alignas(16) int8_t d[kSlices][16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      int8_t q[kSlices];
      digits(P[nu * ldk + kb * 32 + h * 16 + k], e, q);
#pragma unroll
      for (int s = 0; s < kSlices; ++s) d[s][k] = q[s];
    }
    store_row<kRowsB>(dst, t, h, d);
  }
}

// FP64 density matrix (ldk x ldk) from the padded C (kpad x ldc) on CUDA cores:
// small next to the grid work (nbas^2 nocc).
__global__ void k_oz_pmat(const double* __restrict__ C, const double* __restrict__ occ, int64_t ldc, int kpad,
                          int64_t nbas, int64_t ldk, double* __restrict__ P) {
  const int64_t i = (int64_t)blockIdx.y * 16 + threadIdx.y, j = (int64_t)blockIdx.x * 16 + threadIdx.x;
  if (i >= ldk || j >= ldk) return;
  double s = 0.0;
  if (i < nbas && j < nbas)
    for (int k = 0; k < kpad; ++k) s += C[(int64_t)k * ldc + i] * occ[k] * C[(int64_t)k * ldc + j];
  P[i * ldk + j] = s;
}

// ---------------------------------------------------------------------------
// tensor-core pipeline shared by the two contraction kernels
// ---------------------------------------------------------------------------
struct OzSmem {
  alignas(1024) int8_t a[kStages][kOpA];
  alignas(1024) int8_t b[kStages][kOpB];
  double red[4][128];   // density: partial sums of the second column half
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t acc_full;
  uint64_t acc_empty;
  uint32_t tslot;
};
static_assert(sizeof(OzSmem) + 1024 <= tc::kWholeSmSmem, "OzSmem");

__device__ __forceinline__ void oz_mma_step(uint32_t tbase, const int8_t* a, const int8_t* b, bool first) {
  const uint32_t idesc = tc::idesc_s8(kRowsA, kRowsB);
  const uint32_t abase = tc::smem_u32(a), bbase = tc::smem_u32(b);
#pragma unroll
  for (int q = 0; q < kPairs; ++q) {
    const int s = c_oz_pairs[q][0], t = c_oz_pairs[q][1], g = c_oz_pairs[q][2];
    const uint64_t ad = tc::smem_desc(abase + s * kBlkA, 128, 256);
    const uint64_t bd = tc::smem_desc(bbase + t * kBlkB, 128, 256);
    tc::mma_s8(tbase + g * kRowsB, ad, bd, idesc, !(first && pair_leads(q)));
  }
}

// this thread's row of the kGroups accumulators, columns c0..c0+15, combined
// exactly in 64-bit integers: x = sum_g D_g 2^(28-7g) = 2^40 * sum_g 2^(-12-7g) D_g
// (|D_0| < 2^31, so |x| < 2^60), then converted once to FP64.
__device__ __forceinline__ void oz_read16(uint32_t trow, int c0, double (&x)[16]) {
  float v[kGroups][16];
#pragma unroll
  for (int g = 0; g < kGroups; ++g) tc::tmem_ld16(trow + g * kRowsB + c0, v[g]);
  tc::tmem_ld_wait();
#pragma unroll
  for (int g = 0; g < kGroups; ++g) tc::tmem_regs_ready(v[g]);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    long long acc = 0;
#pragma unroll
    for (int g = 0; g < kGroups; ++g) acc += (long long)__float_as_int(v[g][j]) << (7 * (kGroups - 1 - g));
    x[j] = (double)acc;
  }
}


// ---------------------------------------------------------------------------
// G1: density.  CTA = 128 points (TMEM lane = point).  For each 96-wide tile
// of functions nu: X = phi^T P over all K = functions mu, then
// rho += sum_nu X phi, grad rho += 2 sum_nu X grad phi (FP64).
// Warps 0-7 epilogue (warp w: lanes 32(w%4).., columns 48(w/4)..), warp 8
// producer, warp 9 MMA issuer.
// ---------------------------------------------------------------------------
constexpr int kDensThreads = tc::kWholeSmThreads;  // warps 10-15 idle

template <bool GGA>
__global__ void __launch_bounds__(kDensThreads, 1)
    k_oz_density(const int8_t* __restrict__ tA, const int8_t* __restrict__ tB, int nks, int nnb,
                 const int* __restrict__ e_pt, const int* __restrict__ e_P, const double* __restrict__ phi,
                 const double* __restrict__ gx, const double* __restrict__ gy, const double* __restrict__ gz,
                 int64_t ldp, double* __restrict__ rho, double* __restrict__ grx, double* __restrict__ gry,
                 double* __restrict__ grz, int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  OzSmem& S = *reinterpret_cast<OzSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int pb = blockIdx.x;
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&S.full[s], 1);
      tc::mbar_init(&S.empty[s], 1);
    }
    tc::mbar_init(&S.acc_full, 1);
    tc::mbar_init(&S.acc_empty, 256);
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  const int total = nnb * nks;
  bool ok = true;
  double r_acc = 0.0, g_acc[3] = {0.0, 0.0, 0.0};
  if (warp == 8) {
    if (lane == 0) {  // producer
      for (int it = 0; it < total && ok; ++it) {
        const int s = it % kStages, nb = it / nks, kb = it % nks;
        if (it >= kStages && !tc::mbar_wait(&S.empty[s], ((it / kStages) - 1) & 1)) ok = false;
        if (!ok) break;
        tc::mbar_expect_tx(&S.full[s], kOpA + kOpB);
        tc::bulk_g2s(S.a[s], tA + ((int64_t)pb * nks + kb) * kOpA, kOpA, &S.full[s]);
        tc::bulk_g2s(S.b[s], tB + ((int64_t)nb * nks + kb) * kOpB, kOpB, &S.full[s]);
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 9) {
    if (lane == 0) {  // MMA issuer
      int it = 0;
      for (; it < total && ok; ++it) {
        const int s = it % kStages, nb = it / nks, kb = it % nks;
        if (kb == 0 && nb > 0 && !tc::mbar_wait(&S.acc_empty, (nb - 1) & 1)) ok = false;
        if (ok && !tc::mbar_wait(&S.full[s], (it / kStages) & 1)) ok = false;
        if (!ok) break;
        tc::fence_after_sync();
        oz_mma_step(tbase, S.a[s], S.b[s], kb == 0);
        tc::mma_commit(&S.empty[s]);
        if (kb == nks - 1) tc::mma_commit(&S.acc_full);
      }
      if (!ok) {
        atomicExch(err, 1);
        // release the epilogue warps of the remaining tiles (their data is discarded)
        for (int nb = it / nks; nb < nnb; ++nb) tc::mma_commit(&S.acc_full);
      }
    }
  } else if (warp >= 10) {
    // idle: the CTA holds the whole SM
  } else {  // epilogue: thread owns point pb*128 + row, columns half*48 .. +48
    const int row = (warp & 3) * 32 + lane, half = warp >> 2;
    const int64_t p = (int64_t)pb * 128 + row;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16);
    const int ea = e_pt[p];
    const double rs = pow2(ea + kCombShift);  // row scale, applied once per term
    for (int nb = 0; nb < nnb; ++nb) {
      if (!tc::mbar_wait_warp(&S.acc_full, nb & 1)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      for (int c0 = half * 48; c0 < half * 48 + 48; c0 += 16) {
        double x[16];
        oz_read16(trow, c0, x);
        // two halves of 8 columns: the 4 x 8 FP64 loads of a half are in flight together
#pragma unroll
        for (int hh = 0; hh < 16; hh += 8) {
          const int64_t nu0 = (int64_t)nb * kRowsB + c0 + hh;
          double v[8], w0[8], w1[8], w2[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            v[j] = __ldg(phi + (nu0 + j) * ldp + p);
            if (GGA) {
              w0[j] = __ldg(gx + (nu0 + j) * ldp + p);
              w1[j] = __ldg(gy + (nu0 + j) * ldp + p);
              w2[j] = __ldg(gz + (nu0 + j) * ldp + p);
            }
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double X = x[hh + j] * (rs * pow2(__ldg(e_P + nu0 + j)));
            r_acc += X * v[j];
            if (GGA) {
              g_acc[0] += X * w0[j];
              g_acc[1] += X * w1[j];
              g_acc[2] += X * w2[j];
            }
          }
        }
      }
      tc::fence_before_sync();
      tc::mbar_arrive(&S.acc_empty);
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
    const int64_t p = (int64_t)pb * 128 + row;
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
// Z[f][p] = A[p] phi[f][p] (+ B[p] . grad phi[f][p]) in FP64, and the largest
// |Z| of each function (block per (function row, point slab)).
// ---------------------------------------------------------------------------
template <bool GGA>
__global__ void __launch_bounds__(256) k_oz_zbuild(int64_t ldp, const double* __restrict__ phi,
                                                   const double* __restrict__ gx, const double* __restrict__ gy,
                                                   const double* __restrict__ gz, const double* __restrict__ A,
                                                   const double* __restrict__ Bx, const double* __restrict__ By,
                                                   const double* __restrict__ Bz, double* __restrict__ Z,
                                                   unsigned long long* __restrict__ zmax,
                                                   unsigned long long* __restrict__ fmax_) {
  const int64_t f = blockIdx.y;
  const int64_t base = f * ldp;
  double mz = 0.0, mf = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < ldp; p += (int64_t)gridDim.x * blockDim.x) {
    const double v = phi[base + p];
    double z = A[p] * v;
    if (GGA) z += Bx[p] * gx[base + p] + By[p] * gy[base + p] + Bz[p] * gz[base + p];
    Z[base + p] = z;
    mz = fmax(mz, fabs(z));
    mf = fmax(mf, fabs(v));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mz = fmax(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    mf = fmax(mf, __shfl_xor_sync(0xffffffffu, mf, o));
  }
  __shared__ double red[2][8];
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = mz;
    red[1][threadIdx.x >> 5] = mf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < 8; ++i) {
      a = fmax(a, red[0][i]);
      b = fmax(b, red[1][i]);
    }
    if (a > 0.0) atomicMax(zmax + f, (unsigned long long)__double_as_longlong(a));
    if (b > 0.0) atomicMax(fmax_ + f, (unsigned long long)__double_as_longlong(b));
  }
}

// ---------------------------------------------------------------------------
// G2: ham tiles.  grid = (tiles, splits).  ham_IJ = sum_p Z_I(p) phi_J(p)
// (I: 128 functions, J: 96 functions) over the split's points; the FP64
// result is added to the CTA's own partial tile.
// ---------------------------------------------------------------------------
constexpr int kVThreads = tc::kWholeSmThreads;  // warps 6-15 idle

__global__ void __launch_bounds__(kVThreads, 1)
    k_oz_vpot(const int8_t* __restrict__ tZ, const int8_t* __restrict__ tP, int nks, int ks_per_split, int ntb,
              const int* __restrict__ e_Z, const int* __restrict__ e_fn, int ntiles, double* __restrict__ vpart,
              int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  OzSmem& S = *reinterpret_cast<OzSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ti = blockIdx.x / ntb, tj = blockIdx.x % ntb;
  const int kb0 = blockIdx.y * ks_per_split;
  const int kb1 = min(nks, kb0 + ks_per_split);
  const int total = kb1 - kb0;
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&S.full[s], 1);
      tc::mbar_init(&S.empty[s], 1);
    }
    tc::mbar_init(&S.acc_full, 1);
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  bool ok = true;
  if (warp == 4) {
    if (lane == 0) {
      for (int it = 0; it < total && ok; ++it) {
        const int s = it % kStages, kb = kb0 + it;
        if (it >= kStages && !tc::mbar_wait(&S.empty[s], ((it / kStages) - 1) & 1)) ok = false;
        if (!ok) break;
        tc::mbar_expect_tx(&S.full[s], kOpA + kOpB);
        tc::bulk_g2s(S.a[s], tZ + ((int64_t)ti * nks + kb) * kOpA, kOpA, &S.full[s]);
        tc::bulk_g2s(S.b[s], tP + ((int64_t)tj * nks + kb) * kOpB, kOpB, &S.full[s]);
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      for (int it = 0; it < total && ok; ++it) {
        const int s = it % kStages;
        if (!tc::mbar_wait(&S.full[s], (it / kStages) & 1)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        oz_mma_step(tbase, S.a[s], S.b[s], it == 0);
        tc::mma_commit(&S.empty[s]);
      }
      tc::mma_commit(&S.acc_full);  // also on failure: lets the epilogue wind down
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp >= 6) {
    // idle: the CTA holds the whole SM
  } else {
    const bool done = tc::mbar_wait_warp(&S.acc_full, 0);
    if (!done) atomicExch(err, 1);
    tc::fence_after_sync();
    if (done && total > 0) {
      const int r = tid;  // row of the tile = function ti*128 + r
      const int ea = e_Z[ti * kRowsA + r];
      const uint32_t trow = tbase + ((uint32_t)(warp * 32) << 16);
      double* out = vpart + ((int64_t)blockIdx.y * ntiles + blockIdx.x) * (kRowsA * kRowsB) + (int64_t)r * kRowsB;
      for (int c0 = 0; c0 < kRowsB; c0 += 16) {
        double x[16];
        oz_read16(trow, c0, x);
#pragma unroll
        for (int j = 0; j < 16; ++j) out[c0 + j] += x[j] * pow2(ea + kCombShift + __ldg(e_fn + tj * kRowsB + c0 + j));
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

// V(k, j), k <= j, from the 128 x 96 ham tiles: GGA ham(k,j) + ham(j,k); LDA ham(k,j)
__device__ __forceinline__ int64_t ham_off(int64_t r, int64_t c, int ntb) {
  return ((r / kRowsA) * ntb + (c / kRowsB)) * (int64_t)(kRowsA * kRowsB) + (r % kRowsA) * kRowsB + (c % kRowsB);
}

__global__ void k_oz_pack(const double* __restrict__ vpart, int ntb, int ntiles, int nsplit, int64_t nbas, int ispin,
                          int spin, bool gga, double* __restrict__ ham) {
  const int64_t len = nbas * (nbas + 1) / 2;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < len;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > idx) --j;
    while ((j + 1) * (j + 2) / 2 <= idx) ++j;
    const int64_t k = idx - j * (j + 1) / 2;
    const int64_t o1 = ham_off(k, j, ntb), o2 = ham_off(j, k, ntb);
    double v = 0.0;
    for (int s = 0; s < nsplit; ++s) {
      const double* vs = vpart + (int64_t)s * ntiles * (kRowsA * kRowsB);
      v += vs[o1];
      if (gga) v += vs[o2];
    }
    ham[spin + (int64_t)ispin * idx] = v;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int64_t mixed_row_align() { return kAlignFn; }

int mixed_create(MixedState** out, const BuildArgs& a, int64_t nbas, bool gga, int precision, std::string& err) {
  *out = nullptr;
  if (precision != PGXC_PREC_MIXED_INT8) {
    err = "unsupported mixed-precision mode";
    return PGXC_ENOTSUP;
  }
  MixedState* m = new MixedState();
  m->nbas = nbas;
  m->gga = gga;
  m->ldk = round_up(nbas, kAlignFn);
  m->ldp = a.ldp;
  auto fail = [&](cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    mixed_destroy(m);
    return e == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA;
  };
  if (a.ldp % 128) {
    err = "chunk length must be a multiple of 128 points";
    mixed_destroy(m);
    return PGXC_EINVAL;
  }
  const size_t plane = (size_t)m->ldk * m->ldp;
  cudaError_t e;
  if ((e = mx_alloc(m, &m->phi, plane)) || (e = mx_alloc(m, &m->Z, plane))) return fail(e, "cudaMalloc");
  if (gga && ((e = mx_alloc(m, &m->gx, plane)) || (e = mx_alloc(m, &m->gy, plane)) ||
              (e = mx_alloc(m, &m->gz, plane))))
    return fail(e, "cudaMalloc");
  // rows nbas..ldk-1 are never written: zero once
  if ((e = cudaMemset(m->phi, 0, plane * 8)) || (e = cudaMemset(m->Z, 0, plane * 8))) return fail(e, "cudaMemset");
  if (gga && ((e = cudaMemset(m->gx, 0, plane * 8)) || (e = cudaMemset(m->gy, 0, plane * 8)) ||
              (e = cudaMemset(m->gz, 0, plane * 8))))
    return fail(e, "cudaMemset");
  if ((e = mx_alloc(m, &m->tA1, plane * kSlices)) || (e = mx_alloc(m, &m->tZ, plane * kSlices)) ||
      (e = mx_alloc(m, &m->tP2, plane * kSlices)) ||
      (e = mx_alloc(m, &m->tB1, (size_t)m->ldk * m->ldk * kSlices)) ||
      (e = mx_alloc(m, &m->P, (size_t)m->ldk * m->ldk)))
    return fail(e, "cudaMalloc");
  if ((e = mx_alloc(m, &m->e_pt, (size_t)m->ldp)) || (e = mx_alloc(m, &m->e_P, (size_t)m->ldk)) ||
      (e = mx_alloc(m, &m->e_Z, (size_t)m->ldk)) || (e = mx_alloc(m, &m->e_fn, (size_t)m->ldk)) ||
      (e = mx_alloc(m, &m->zmax, (size_t)m->ldk)) || (e = mx_alloc(m, &m->fmax, (size_t)m->ldk)))
    return fail(e, "cudaMalloc");
  if ((e = mx_alloc(m, &m->err, 1)) || (e = cudaMemset(m->err, 0, sizeof(int)))) return fail(e, "cudaMalloc");
  m->nta = (int)(m->ldk / kRowsA);
  m->ntb = (int)(m->ldk / kRowsB);
  m->ntiles = m->nta * m->ntb;
  // splits of the chunk's K steps: enough CTAs for the SMs, and at most
  // 65536 points per split so that |D_g| <= 5*4096*K stays below 2^31
  const int nks = (int)(m->ldp / kKStep);
  int ns = std::max(1, (148 + m->ntiles - 1) / m->ntiles);
  while ((nks + ns - 1) / ns > 65536 / kKStep) ++ns;
  ns = std::min(ns, nks);
  m->ks_per_split = (nks + ns - 1) / ns;
  m->nsplit = (nks + m->ks_per_split - 1) / m->ks_per_split;
  if ((e = mx_alloc(m, &m->vpart, (size_t)m->nsplit * m->ntiles * kRowsA * kRowsB))) return fail(e, "cudaMalloc");
  const int smem = tc::kWholeSmSmem;  // >= sizeof(OzSmem) + 1024 (base alignment)
  if ((e = cudaFuncSetAttribute(k_oz_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) ||
      (e = cudaFuncSetAttribute(k_oz_density<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) ||
      (e = cudaFuncSetAttribute(k_oz_vpot, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)))
    return fail(e, "cudaFuncSetAttribute");
  *out = m;
  return PGXC_OK;
}

void mixed_destroy(MixedState* m) {
  if (!m) return;
  for (void* p : m->allocs) cudaFree(p);
  delete m;
}

int mixed_error_flag(MixedState* m, cudaStream_t st, int* flag) {
  cudaMemcpyAsync(flag, m->err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemsetAsync(m->err, 0, sizeof(int), st);
  return cudaStreamSynchronize(st) == cudaSuccess ? PGXC_OK : PGXC_ECUDA;
}

int mixed_prepare(MixedState* m, const BuildArgs& a, int nocc, cudaStream_t st) {
  const int kpad = (int)round_up(std::max(nocc, 1), 16);
  dim3 b2(16, 16), g2((unsigned)(m->ldk / 16), (unsigned)(m->ldk / 16));
  k_oz_pmat<<<g2, b2, 0, st>>>(a.C, a.occ, a.ldc, kpad, m->nbas, m->ldk, m->P);
  k_oz_rowexp_P<<<(unsigned)m->ldk, 256, 0, st>>>(m->P, m->ldk, m->e_P);
  const int nks = (int)(m->ldk / kKStep);
  k_oz_quant_P<<<dim3((unsigned)(m->ldk / kRowsB), (unsigned)nks), kBlock4(kRowsB), 0, st>>>(m->P, m->ldk, m->e_P, nks,
                                                                                  m->tB1);
  cudaMemsetAsync(m->vpart, 0, sizeof(double) * m->nsplit * m->ntiles * kRowsA * kRowsB, st);
  return 3;
}

// A density matrix given by the caller (ldc x ldc, nbas x nbas used) -> the padded copy.
__global__ void k_oz_copy_P(const double* __restrict__ Pin, int64_t ldc, int64_t nbas, int64_t ldk,
                            double* __restrict__ P) {
  const int64_t i = (int64_t)blockIdx.y * 16 + threadIdx.y, j = (int64_t)blockIdx.x * 16 + threadIdx.x;
  if (i >= ldk || j >= ldk) return;
  P[i * ldk + j] = (i < nbas && j < nbas) ? Pin[i * ldc + j] : 0.0;
}

int mixed_prepare_P(MixedState* m, const double* P, int64_t ldc, cudaStream_t st) {
  dim3 b2(16, 16), g2((unsigned)(m->ldk / 16), (unsigned)(m->ldk / 16));
  k_oz_copy_P<<<g2, b2, 0, st>>>(P, ldc, m->nbas, m->ldk, m->P);
  k_oz_rowexp_P<<<(unsigned)m->ldk, 256, 0, st>>>(m->P, m->ldk, m->e_P);
  const int nks = (int)(m->ldk / kKStep);
  k_oz_quant_P<<<dim3((unsigned)(m->ldk / kRowsB), (unsigned)nks), kBlock4(kRowsB), 0, st>>>(m->P, m->ldk, m->e_P, nks,
                                                                                  m->tB1);
  cudaMemsetAsync(m->vpart, 0, sizeof(double) * m->nsplit * m->ntiles * kRowsA * kRowsB, st);
  return 3;
}

int mixed_basis(MixedState* m, const BuildArgs& a, int64_t p0, int64_t nvalid, bool gga, cudaStream_t st) {
  launch_basis(a, a.px, a.py, a.pz, p0, nvalid, m->ldp, m->phi, gga ? m->gx : nullptr, m->gy, m->gz, st);
  const int nksf = (int)(m->ldk / kKStep);
  k_oz_quant_pts<<<(unsigned)(m->ldp / 128), 128, 0, st>>>(m->phi, m->ldp, m->nbas, nksf, m->e_pt, m->tA1);
  return 5;
}

int mixed_density(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st) {
  const int smem = tc::kWholeSmSmem;  // >= sizeof(OzSmem) + 1024 (base alignment)
  const int nks = (int)(m->ldk / kKStep), nnb = (int)(m->ldk / kRowsB);
  dim3 grid((unsigned)(m->ldp / 128));
  if (gga)
    k_oz_density<true><<<grid, kDensThreads, smem, st>>>(m->tA1, m->tB1, nks, nnb, m->e_pt, m->e_P, m->phi, m->gx,
                                                         m->gy, m->gz, m->ldp, a.rho, a.grx, a.gry, a.grz, m->err);
  else
    k_oz_density<false><<<grid, kDensThreads, smem, st>>>(m->tA1, m->tB1, nks, nnb, m->e_pt, m->e_P, m->phi, nullptr,
                                                          nullptr, nullptr, m->ldp, a.rho, nullptr, nullptr, nullptr,
                                                          m->err);
  return 1;
}

int mixed_potential(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1) {
  cudaMemsetAsync(m->zmax, 0, sizeof(unsigned long long) * m->ldk, st);
  cudaMemsetAsync(m->fmax, 0, sizeof(unsigned long long) * m->ldk, st);
  dim3 gz((unsigned)std::min<int64_t>(64, (m->ldp + 255) / 256), (unsigned)m->nbas);
  if (gga)
    k_oz_zbuild<true><<<gz, 256, 0, st>>>(m->ldp, m->phi, m->gx, m->gy, m->gz, a.A, a.Bx, a.By, a.Bz, m->Z, m->zmax,
                                          m->fmax);
  else
    k_oz_zbuild<false><<<gz, 256, 0, st>>>(m->ldp, m->phi, nullptr, nullptr, nullptr, a.A, nullptr, nullptr, nullptr,
                                           m->Z, m->zmax, m->fmax);
  const unsigned ne = (unsigned)((m->ldk + 255) / 256);
  k_oz_fexp<<<ne, 256, 0, st>>>(m->zmax, m->ldk, m->e_Z);
  k_oz_fexp<<<ne, 256, 0, st>>>(m->fmax, m->ldk, m->e_fn);
  const int nks = (int)(m->ldp / kKStep);
  k_oz_quant_fn<kRowsA><<<dim3((unsigned)m->nta, (unsigned)nks), kBlock4(kRowsA), 0, st>>>(m->Z, m->ldp, m->e_Z, nks, m->tZ);
  k_oz_quant_fn<kRowsB><<<dim3((unsigned)m->ntb, (unsigned)nks), kBlock4(kRowsB), 0, st>>>(m->phi, m->ldp, m->e_fn, nks,
                                                                                 m->tP2);
  cudaEventRecord(k0, st);
  const int smem = tc::kWholeSmSmem;  // >= sizeof(OzSmem) + 1024 (base alignment)
  k_oz_vpot<<<dim3((unsigned)m->ntiles, (unsigned)m->nsplit), kVThreads, smem, st>>>(
      m->tZ, m->tP2, nks, m->ks_per_split, m->ntb, m->e_Z, m->e_fn, m->ntiles, m->vpart, m->err);
  cudaEventRecord(k1, st);
  return 6;
}

int mixed_pack(MixedState* m, const BuildArgs&, int64_t nbas, int ispin, int spin, double* ham, cudaStream_t st) {
  const int64_t len = nbas * (nbas + 1) / 2;
  const unsigned nb = (unsigned)std::min<int64_t>((len + 255) / 256, 148 * 8);
  k_oz_pack<<<nb, 256, 0, st>>>(m->vpart, m->ntb, m->ntiles, m->nsplit, nbas, ispin, spin, m->gga, ham);
  return 1;
}

}  // namespace pgxc
