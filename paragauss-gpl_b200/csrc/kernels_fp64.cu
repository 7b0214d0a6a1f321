// kernels_fp64.cu -- the FP64 (drop-in) XC-build kernels.
//
// Per build (one SCF cycle):
//   k_scale_occ    C_occ = C * occ                          (P = C diag(occ) C^T)
//   k_pmat         P = C^T-layout GEMM on DMMA
// per grid chunk of CH points:
//   k_basis        phi, grad phi (FP64)                      [K1]
//   k_density      X = phi^T P on DMMA, fused rho = sum X*phi, grad rho = 2 sum X*grad phi   [K3]
//   k_functional   f, df/drho, df/dgamma; A, B; E_xc, N_el block partials   [K2]
//   k_zbuild       Z = A phi (+ B . grad phi)
//   k_vpot         V tiles += sum_p (Z_I phi_J [+ phi_I Z_J]) on DMMA, split over points   [K4]
// after the last chunk:
//   k_pack         V -> packed upper triangle (tristore order)
//
// The density is formed from P rather than from the occupied orbitals as the
// reference does (density_calc_nl, modules/density_calc_module.f90:1447-1576);
// the two are equal, P = C diag(occ) C^T, up to rounding.
#include <cstdint>
#include <cuda_runtime.h>

#include "basis.cuh"
#include "dgemm.cuh"
#include "pgxc_common.cuh"
#include "kernels.h"
#include "xc_functional.cuh"

namespace pgxc {

// ---------------------------------------------------------------------------
// K1: basis functions, one launch per angular momentum (k_basis_l, basis.cuh)
// ---------------------------------------------------------------------------
template <int L>
static void launch_basis_one_l(const BuildArgs& a, const double* px, const double* py, const double* pz, int64_t p0,
                               int64_t nvalid, int64_t ld, double* phi, double* gx, double* gy, double* gz,
                               cudaStream_t st) {
  if (a.nshl[L] == 0) return;
  dim3 grid((unsigned)((ld + 127) / 128), (unsigned)a.nshl[L]);
  if (gx)
    k_basis_l<L, true><<<grid, 128, 0, st>>>(a.shells, a.shl[L], a.atoms, a.exps, a.norms, a.contr, a.rng, a.sa, px,
                                                     py, pz, p0, nvalid, ld, phi, gx, gy, gz);
  else
    k_basis_l<L, false><<<grid, 128, 0, st>>>(a.shells, a.shl[L], a.atoms, a.exps, a.norms, a.contr, a.rng, a.sa,
                                                      px, py, pz, p0, nvalid, ld, phi, nullptr, nullptr, nullptr);
}

void launch_basis(const BuildArgs& a, const double* px, const double* py, const double* pz, int64_t p0,
                  int64_t nvalid, int64_t ld, double* phi, double* gx, double* gy, double* gz, cudaStream_t st) {
  launch_basis_one_l<0>(a, px, py, pz, p0, nvalid, ld, phi, gx, gy, gz, st);
  launch_basis_one_l<1>(a, px, py, pz, p0, nvalid, ld, phi, gx, gy, gz, st);
  launch_basis_one_l<2>(a, px, py, pz, p0, nvalid, ld, phi, gx, gy, gz, st);
  launch_basis_one_l<3>(a, px, py, pz, p0, nvalid, ld, phi, gx, gy, gz, st);
}

void launch_basis_f64(const BuildArgs& a, int64_t p0, int64_t nvalid, bool grad, cudaStream_t st) {
  launch_basis(a, a.px, a.py, a.pz, p0, nvalid, a.ldp, a.phi, grad ? a.gx : nullptr, a.gy, a.gz, st);
}

// basis on arbitrary points (pgxc_orbital_calculate): same kernels, caller arrays
void launch_basis_points_f64(const BuildArgs& a, const double* px, const double* py, const double* pz, int64_t n,
                             int64_t ld, double* phi, double* gx, double* gy, double* gz, cudaStream_t st) {
  launch_basis(a, px, py, pz, 0, n, ld, phi, gx, gy, gz, st);
}

// ---------------------------------------------------------------------------
// Density matrix: Cocc[j][mu] = occ_j C[j][mu];  P = sum_j C[j][mu] Cocc[j][nu]
// ---------------------------------------------------------------------------
__global__ void k_scale_occ(const double* __restrict__ C, const double* __restrict__ occ, int64_t ldc, int nocc,
                            double* __restrict__ Cocc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ldc * nocc) return;
  const int j = (int)(i / ldc);
  Cocc[i] = C[i] * occ[j];
}

__global__ void __launch_bounds__(kGemmThreads) k_pmat(const double* __restrict__ C, const double* __restrict__ Cocc,
                                                      int64_t ldc, int64_t kpad, double* __restrict__ P) {
  extern __shared__ double smem[];
  const int64_t m0 = (int64_t)blockIdx.x * 64, n0 = (int64_t)blockIdx.y * 64;
  Acc acc;
  acc.zero();
  gemm_tile<false, false>(acc, C, ldc, m0, Cocc, ldc, n0, 0, kpad, smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t r = m0 + wm0 + i * 8 + (lane >> 2);
        const int64_t c = n0 + wn0 + j * 8 + 2 * (lane & 3) + e;
        P[r * ldc + c] = acc.v[i][j][e];
      }
}

void launch_pmat_f64(const BuildArgs& a, int64_t kpad, cudaStream_t st) {
  const int64_t n = a.ldc * kpad;
  k_scale_occ<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.C, a.occ, a.ldc, (int)kpad, a.Cocc);
  constexpr int smem = gemm_smem_bytes<false, false>();
  cudaFuncSetAttribute(k_pmat, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  dim3 grid((unsigned)(a.ldc / 64), (unsigned)(a.ldc / 64));
  k_pmat<<<grid, kGemmThreads, smem, st>>>(a.C, a.Cocc, a.ldc, kpad, a.P);
}

// ---------------------------------------------------------------------------
// K3: X = phi^T P (points x functions), fused with the row reductions
//   rho[p] = sum_nu X[p][nu] phi[nu][p],  grad rho[p] = 2 sum_nu X[p][nu] grad phi[nu][p].
// One CTA owns 64 points and loops over all 64-wide function tiles.
// ---------------------------------------------------------------------------
template <bool GGA>
__global__ void __launch_bounds__(kGemmThreads) k_density(const double* __restrict__ phi, const double* __restrict__ gx,
                                                         const double* __restrict__ gy, const double* __restrict__ gz,
                                                         int64_t ldp, const double* __restrict__ P, int64_t ldc,
                                                         double* __restrict__ rho, double* __restrict__ grx,
                                                         double* __restrict__ gry, double* __restrict__ grz) {
  extern __shared__ double smem[];
  const int64_t m0 = (int64_t)blockIdx.x * 64;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
  double rp[4][2] = {}, gp[3][4][2] = {};
  for (int64_t n0 = 0; n0 < ldc; n0 += 64) {
    Acc acc;
    acc.zero();
    gemm_tile<false, false>(acc, phi, ldp, m0, P, ldc, n0, 0, ldc, smem);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t r = m0 + wm0 + i * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int64_t c = n0 + wn0 + j * 8 + 2 * (lane & 3) + e;
          const double x = acc.v[i][j][e];
          rp[i][e] += x * phi[c * ldp + r];
          if (GGA) {
            gp[0][i][e] += x * gx[c * ldp + r];
            gp[1][i][e] += x * gy[c * ldp + r];
            gp[2][i][e] += x * gz[c * ldp + r];
          }
        }
    }
  }
  // reduce the 4 lanes of a row, then the two column-warps through smem
  double* red = smem;  // [2 warps-n][4 quantities][64 rows]
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double v[4];
    v[0] = rp[i][0] + rp[i][1];
    if (GGA) {
      v[1] = gp[0][i][0] + gp[0][i][1];
      v[2] = gp[1][i][0] + gp[1][i][1];
      v[3] = gp[2][i][0] + gp[2][i][1];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q > 0 && !GGA) break;
      v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
      v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
      if ((lane & 3) == 0) red[((warp & 1) * 4 + q) * 64 + wm0 + i * 8 + (lane >> 2)] = v[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    const int r = threadIdx.x;
    rho[m0 + r] = red[0 * 64 + r] + red[4 * 64 + r];
    if (GGA) {
      grx[m0 + r] = 2.0 * (red[1 * 64 + r] + red[5 * 64 + r]);
      gry[m0 + r] = 2.0 * (red[2 * 64 + r] + red[6 * 64 + r]);
      grz[m0 + r] = 2.0 * (red[3 * 64 + r] + red[7 * 64 + r]);
    }
  }
}

void launch_density_f64(const BuildArgs& a, bool gga, cudaStream_t st) {
  constexpr int smem = gemm_smem_bytes<false, false>();
  dim3 grid((unsigned)(a.ldp / 64));
  if (gga) {
    cudaFuncSetAttribute(k_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_density<true><<<grid, kGemmThreads, smem, st>>>(a.phi, a.gx, a.gy, a.gz, a.ldp, a.P, a.ldc, a.rho, a.grx,
                                                      a.gry, a.grz);
  } else {
    cudaFuncSetAttribute(k_density<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_density<false><<<grid, kGemmThreads, smem, st>>>(a.phi, nullptr, nullptr, nullptr, a.ldp, a.P, a.ldc, a.rho,
                                                       nullptr, nullptr, nullptr);
  }
}

// ---------------------------------------------------------------------------
// K2: functional per point.  Writes A = w df/drho (VWN) or w df/drho / 2
// (PBE), B = 2 w df/dgamma grad rho (PBE), and per-block partial sums of
// w*f and w*rho (exc_int, charge_int).  rho is clamped at 0: in P form it can
// round to tiny negative values where the reference's sum of squares is +0.
// ---------------------------------------------------------------------------
template <bool GGA>
__global__ void __launch_bounds__(256) k_functional(XcConst K, int64_t p0, int64_t nvalid, int64_t n, const double* __restrict__ w,
                                                    const double* __restrict__ rho, const double* __restrict__ grx,
                                                    const double* __restrict__ gry, const double* __restrict__ grz,
                                                    double* __restrict__ A, double* __restrict__ Bx,
                                                    double* __restrict__ By, double* __restrict__ Bz,
                                                    double* __restrict__ partial) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, q = 0.0;
  if (p < n) {
    const double wt = (p < nvalid) ? w[p0 + p] : 0.0;
    const double r = fmax(rho[p], 0.0);
    if (GGA) {
      const double g0 = grx[p], g1 = gry[p], g2 = grz[p];
      const double g = g0 * g0 + g1 * g1 + g2 * g2;
      double f, fr, fg;
      xc_gga(K, r, g, f, fr, fg);
      A[p] = 0.5 * fr * wt;
      const double b = wt * 2.0 * fg;
      Bx[p] = b * g0;
      By[p] = b * g1;
      Bz[p] = b * g2;
      e = f * wt;
    } else {
      double f, fr;
      xc_vwn(K, r, f, fr);
      A[p] = fr * wt;
      e = f * wt;
    }
    q = r * wt;
  }
  // fixed-order block reduction (deterministic; blockDim a power of two <= 256)
  __shared__ double se[256], sq[256];
  se[threadIdx.x] = e;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = se[0];
    partial[2 * blockIdx.x + 1] = sq[0];
  }
}

// Sum the block partials in a fixed order and Kahan-add them into acc[4]
// = {E, E compensation, N, N compensation}: compensated across chunks.
__global__ void k_sum_partials(const double* __restrict__ partial, int nblocks, double* __restrict__ acc) {
  __shared__ double se[256], sq[256];
  double e = 0.0, q = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += 256) {
    e += partial[2 * i];
    q += partial[2 * i + 1];
  }
  se[threadIdx.x] = e;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double vals[2] = {se[0], sq[0]};
    for (int k = 0; k < 2; ++k) {
      const double y = vals[k] - acc[2 * k + 1];
      const double t = acc[2 * k] + y;
      acc[2 * k + 1] = (t - acc[2 * k]) - y;
      acc[2 * k] = t;
    }
  }
}

// Open shell (ispin = 2).  pa / pb hold the point arrays of spin a / b, each
// as 8 columns of ld: rho, grad rho (x, y, z), A, B (x, y, z).  Per spin s,
// A_s = w df/drho_s (VWN) or w df/drho_s / 2 (PBE) and
// B_s = w (2 df/dgamma_ss grad rho_s + df/dgamma_ab grad rho_s')
// (modules/xc_hamiltonian.f90:1429-1446); partials of w f and w (rho_a + rho_b).
template <bool GGA>
__global__ void __launch_bounds__(256) k_functional2(XcConst K, int64_t p0, int64_t nvalid, int64_t n,
                                                     const double* __restrict__ w, double* __restrict__ pa,
                                                     double* __restrict__ pb, int64_t ld,
                                                     double* __restrict__ partial) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, q = 0.0;
  if (p < n) {
    const double wt = (p < nvalid) ? w[p0 + p] : 0.0;
    const double rho[2] = {fmax(pa[p], 0.0), fmax(pb[p], 0.0)};
    double ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0}, gam[3] = {0, 0, 0};
    if (GGA) {
      for (int c = 0; c < 3; ++c) {
        ga[c] = pa[(1 + c) * ld + p];
        gb[c] = pb[(1 + c) * ld + p];
      }
      gam[0] = ga[0] * ga[0] + ga[1] * ga[1] + ga[2] * ga[2];
      gam[1] = gb[0] * gb[0] + gb[1] * gb[1] + gb[2] * gb[2];
      gam[2] = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
    }
    double f, fr[2], fg[3];
    xc_open<GGA>(K, rho, gam, f, fr, fg);
    if (GGA) {
      pa[4 * ld + p] = 0.5 * fr[0] * wt;
      pb[4 * ld + p] = 0.5 * fr[1] * wt;
      for (int c = 0; c < 3; ++c) {
        pa[(5 + c) * ld + p] = wt * (2.0 * fg[0] * ga[c] + fg[2] * gb[c]);
        pb[(5 + c) * ld + p] = wt * (2.0 * fg[1] * gb[c] + fg[2] * ga[c]);
      }
    } else {
      pa[4 * ld + p] = fr[0] * wt;
      pb[4 * ld + p] = fr[1] * wt;
    }
    e = f * wt;
    q = (rho[0] + rho[1]) * wt;
  }
  __shared__ double se[256], sq[256];
  se[threadIdx.x] = e;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = se[0];
    partial[2 * blockIdx.x + 1] = sq[0];
  }
}

void launch_sum_partials(const double* partial, int nblocks, double* acc, cudaStream_t st) {
  k_sum_partials<<<1, 256, 0, st>>>(partial, nblocks, acc);
}

void launch_functional2_f64(const XcConst& K, const double* w, double* pa, double* pb, int64_t ld, int64_t p0,
                            int64_t nvalid, bool gga, double* partial, double* acc, cudaStream_t st) {
  const unsigned nb = (unsigned)((ld + 255) / 256);
  if (gga) k_functional2<true><<<nb, 256, 0, st>>>(K, p0, nvalid, ld, w, pa, pb, ld, partial);
  else k_functional2<false><<<nb, 256, 0, st>>>(K, p0, nvalid, ld, w, pa, pb, ld, partial);
  k_sum_partials<<<1, 256, 0, st>>>(partial, (int)nb, acc);
}

void launch_functional_f64(const BuildArgs& a, int64_t p0, int64_t nvalid, bool gga, cudaStream_t st) {
  const unsigned nb = (unsigned)((a.ldp + 255) / 256);
  if (gga)
    k_functional<true><<<nb, 256, 0, st>>>(a.xc, p0, nvalid, a.ldp, a.w, a.rho, a.grx, a.gry, a.grz, a.A, a.Bx, a.By,
                                           a.Bz, a.partial);
  else
    k_functional<false><<<nb, 256, 0, st>>>(a.xc, p0, nvalid, a.ldp, a.w, a.rho, nullptr, nullptr, nullptr, a.A, nullptr,
                                            nullptr, nullptr, a.partial);
  k_sum_partials<<<1, 256, 0, st>>>(a.partial, (int)nb, a.acc);
}

// One block per 128-point tile of a set's chunk: partial[2 t], partial[2 t + 1]
// = the tile's sums of w f and w rho (reduced per context by the caller).
void launch_functional_tiles(const BuildArgs& a, int64_t p0, int64_t ntiles, bool gga, cudaStream_t st) {
  const int64_t n = ntiles * 128;
  if (gga)
    k_functional<true><<<(unsigned)ntiles, 128, 0, st>>>(a.xc, p0, n, n, a.w, a.rho, a.grx, a.gry, a.grz, a.A, a.Bx,
                                                         a.By, a.Bz, a.partial);
  else
    k_functional<false><<<(unsigned)ntiles, 128, 0, st>>>(a.xc, p0, n, n, a.w, a.rho, nullptr, nullptr, nullptr, a.A,
                                                          nullptr, nullptr, nullptr, a.partial);
}

// ---------------------------------------------------------------------------
// Z[f][p] = A[p] phi[f][p] (+ B[p] . grad phi[f][p])   (orbs_help, :1479-1482)
// ---------------------------------------------------------------------------
template <bool GGA>
__global__ void k_zbuild(int64_t nf, int64_t ldp, const double* __restrict__ phi, const double* __restrict__ gx,
                         const double* __restrict__ gy, const double* __restrict__ gz, const double* __restrict__ A,
                         const double* __restrict__ Bx, const double* __restrict__ By,
                         const double* __restrict__ Bz, double* __restrict__ Z) {
  const int64_t total = nf * ldp;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i % ldp;
    double z = A[p] * phi[i];
    if (GGA) z += Bx[p] * gx[i] + By[p] * gy[i] + Bz[p] * gz[i];
    Z[i] = z;
  }
}

void launch_zbuild_f64(const BuildArgs& a, bool gga, cudaStream_t st) {
  const unsigned nb = 148 * 16;
  if (gga)
    k_zbuild<true><<<nb, 256, 0, st>>>(a.ldc, a.ldp, a.phi, a.gx, a.gy, a.gz, a.A, a.Bx, a.By, a.Bz, a.Z);
  else
    k_zbuild<false><<<nb, 256, 0, st>>>(a.ldc, a.ldp, a.phi, nullptr, nullptr, nullptr, a.A, nullptr, nullptr,
                                        nullptr, a.Z);
}

// ---------------------------------------------------------------------------
// K4: V tiles.  grid = (n upper tiles, nsplit).  Tile t = (I, J), I <= J;
// split s covers points [s*kspan, (s+1)*kspan).  LDA: V_IJ += sum phi_I Z_J;
// GGA: V_IJ += sum (Z_I phi_J + phi_I Z_J)  (ham + ham^T of :1559-1566).
// Each (split, tile) is owned by one CTA per launch: += is race-free and the
// summation order is fixed.
// ---------------------------------------------------------------------------
template <bool GGA>
__global__ void __launch_bounds__(kGemmThreads) k_vpot(const double* __restrict__ phi, const double* __restrict__ Z,
                                                      int64_t ldp, int64_t kspan, const int2* __restrict__ tiles,
                                                      int ntiles, double* __restrict__ vpart) {
  extern __shared__ double smem[];
  const int2 t = tiles[blockIdx.x];
  const int64_t m0 = (int64_t)t.x * 64, n0 = (int64_t)t.y * 64;
  const int64_t k0 = (int64_t)blockIdx.y * kspan, k1 = k0 + kspan;
  Acc acc;
  acc.zero();
  if (GGA) gemm_tile<true, true>(acc, Z, ldp, m0, phi, ldp, n0, k0, k1, smem);
  gemm_tile<true, true>(acc, phi, ldp, m0, Z, ldp, n0, k0, k1, smem);
  double* out = vpart + ((int64_t)blockIdx.y * ntiles + blockIdx.x) * 64 * 64;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = wm0 + i * 8 + (lane >> 2);
      const int c = wn0 + j * 8 + 2 * (lane & 3);
      double2* o = reinterpret_cast<double2*>(out + r * 64 + c);
      double2 v = *o;
      v.x += acc.v[i][j][0];
      v.y += acc.v[i][j][1];
      *o = v;
    }
}

void launch_vpot_f64(const BuildArgs& a, bool gga, cudaStream_t st) {
  constexpr int smem = gemm_smem_bytes<true, true>();
  dim3 grid((unsigned)a.ntiles, (unsigned)a.nsplit);
  if (gga) {
    cudaFuncSetAttribute(k_vpot<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_vpot<true><<<grid, kGemmThreads, smem, st>>>(a.phi, a.Z, a.ldp, a.kspan, a.tiles, a.ntiles, a.vpart);
  } else {
    cudaFuncSetAttribute(k_vpot<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_vpot<false><<<grid, kGemmThreads, smem, st>>>(a.phi, a.Z, a.ldp, a.kspan, a.tiles, a.ntiles, a.vpart);
  }
}

// ---------------------------------------------------------------------------
// Pack: ham[s + ispin*(j(j+1)/2 + k)] = sum_split V(k, j), k <= j.
// ---------------------------------------------------------------------------
__global__ void k_pack(const double* __restrict__ vpart, const int* __restrict__ tile_of, int nt, int ntiles,
                       int nsplit, int64_t nbas, int ispin, int spin, double* __restrict__ ham) {
  const int64_t len = nbas * (nbas + 1) / 2;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < len;
       idx += (int64_t)gridDim.x * blockDim.x) {
    // invert idx = j(j+1)/2 + k
    int64_t j = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > idx) --j;
    while ((j + 1) * (j + 2) / 2 <= idx) ++j;
    const int64_t k = idx - j * (j + 1) / 2;
    const int I = (int)(k / 64), J = (int)(j / 64);
    const int t = tile_of[I * nt + J];
    const int64_t off = (int64_t)t * 4096 + (k % 64) * 64 + (j % 64);
    double v = 0.0;
    for (int s = 0; s < nsplit; ++s) v += vpart[(int64_t)s * ntiles * 4096 + off];
    ham[spin + (int64_t)ispin * idx] = v;
  }
}

void launch_pack(const BuildArgs& a, int64_t nbas, int ispin, int spin, double* ham, cudaStream_t st) {
  const int64_t len = nbas * (nbas + 1) / 2;
  const unsigned nb = (unsigned)std::min<int64_t>((len + 255) / 256, 148 * 8);
  k_pack<<<nb, 256, 0, st>>>(a.vpart, a.tile_of, a.nt, a.ntiles, a.nsplit, nbas, ispin, spin, ham);
}

}  // namespace pgxc
