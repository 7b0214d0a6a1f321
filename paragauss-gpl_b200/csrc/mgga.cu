// mgga.cu -- the meta-GGA functional step of the screened builds (TPSS,
// M06-L, M06, VSXC).
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"
#include "xc_mgga.cuh"

namespace pgxc {

namespace {

// Per point: rho, grad rho (pt planes 0..3 of each spin), tau = 1/2 (Tx + Ty +
// Tz) (tq planes 0..2 of each spin) -> A = w df/drho_s / 2, B = w (2
// df/dgamma_ss grad rho_s + df/dgamma_ab grad rho_s') (pt planes 4..7), C =
// w df/dtau_s / 4 (tq plane 3): the potential then adds C grad phi_i .
// grad phi_j to the matrix it symmetrises (V = H + H^T), i.e. 1/2 w df/dtau
// grad phi_i . grad phi_j as calc_xcks_nl (xc_hamiltonian.f90:1448-1454,
// :1534-1555).  Partials of w f and w rho as k_functional.
template <int ISPIN>
__global__ void __launch_bounds__(256) k_functional_mgga(int functional, int64_t p0, int64_t nvalid, int64_t n,
                                                         const double* __restrict__ w, double* __restrict__ pt,
                                                         double* __restrict__ tq, int64_t ld,
                                                         double* __restrict__ partial) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, q = 0.0;
  if (p < n) {
    const double wt = (p < nvalid) ? w[p0 + p] : 0.0;
    double rho[2], g[2][3], tau[2];
#pragma unroll
    for (int s = 0; s < ISPIN; ++s) {
      const double* a = pt + 8 * s * ld;
      const double* b = tq + 4 * s * ld;
      rho[s] = fmax(a[p], 0.0);
#pragma unroll
      for (int c = 0; c < 3; ++c) g[s][c] = a[(1 + c) * ld + p];
      tau[s] = fmax(0.5 * (b[p] + b[ld + p] + b[2 * ld + p]), 0.0);
    }
    if (ISPIN == 1) {
      const double gam = g[0][0] * g[0][0] + g[0][1] * g[0][1] + g[0][2] * g[0][2];
      double f, fr, fg, ft;
      mgga::mgga_closed(functional, rho[0], gam, tau[0], f, fr, fg, ft);
      pt[4 * ld + p] = 0.5 * fr * wt;
      const double bb = wt * 2.0 * fg;
#pragma unroll
      for (int c = 0; c < 3; ++c) pt[(5 + c) * ld + p] = bb * g[0][c];
      tq[3 * ld + p] = 0.25 * ft * wt;
      e = f * wt;
      q = rho[0] * wt;
    } else {
      double gam[3] = {0, 0, 0};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gam[0] += g[0][c] * g[0][c];
        gam[1] += g[1][c] * g[1][c];
        gam[2] += g[0][c] * g[1][c];
      }
      double f, fr[2], fg[3], ft[2];
      mgga::mgga_open(functional, rho, gam, tau, f, fr, fg, ft);
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        double* a = pt + 8 * s * ld;
        a[4 * ld + p] = 0.5 * fr[s] * wt;
#pragma unroll
        for (int c = 0; c < 3; ++c) a[(5 + c) * ld + p] = wt * (2.0 * fg[s] * g[s][c] + fg[2] * g[1 - s][c]);
        tq[4 * s * ld + 3 * ld + p] = 0.25 * ft[s] * wt;
      }
      e = f * wt;
      q = (rho[0] + rho[1]) * wt;
    }
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

// The meta-GGA at n points, column-major: rho (ispin), gam (2 ispin - 1),
// tau (ispin) -> f, fr (ispin), fg (2 ispin - 1), ft (ispin).
template <int ISPIN>
__global__ void k_xc_points_mgga(int functional, int64_t n, const double* __restrict__ rho, const double* __restrict__ gam,
                                 const double* __restrict__ tau, double* __restrict__ f, double* __restrict__ fr,
                                 double* __restrict__ fg, double* __restrict__ ft) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (ISPIN == 1) {
    double F, Fr, Fg, Ft;
    mgga::mgga_closed(functional, rho[p], gam[p], tau[p], F, Fr, Fg, Ft);
    f[p] = F;
    fr[p] = Fr;
    fg[p] = Fg;
    ft[p] = Ft;
  } else {
    const double r[2] = {rho[p], rho[p + n]}, g[3] = {gam[p], gam[p + n], gam[p + 2 * n]},
                 t[2] = {tau[p], tau[p + n]};
    double F, Fr[2], Fg[3], Ft[2];
    mgga::mgga_open(functional, r, g, t, F, Fr, Fg, Ft);
    f[p] = F;
    for (int s = 0; s < 2; ++s) {
      fr[p + s * n] = Fr[s];
      ft[p + s * n] = Ft[s];
    }
    for (int c = 0; c < 3; ++c) fg[p + c * n] = Fg[c];
  }
}

}  // namespace

void launch_xc_points_mgga(int functional, int ispin, int64_t n, const double* rho, const double* gam, const double* tau, double* f,
                           double* fr, double* fg, double* ft, cudaStream_t st) {
  const unsigned nb = (unsigned)((n + 127) / 128);
  if (ispin == 1) k_xc_points_mgga<1><<<nb, 128, 0, st>>>(functional, n, rho, gam, tau, f, fr, fg, ft);
  else k_xc_points_mgga<2><<<nb, 128, 0, st>>>(functional, n, rho, gam, tau, f, fr, fg, ft);
}

void launch_functional_mgga(int functional, int ispin, const double* w, double* pt, double* tq, int64_t ld, int64_t p0,
                            int64_t nvalid, double* partial, double* acc, cudaStream_t st) {
  const unsigned nb = (unsigned)((ld + 255) / 256);
  if (ispin == 1) k_functional_mgga<1><<<nb, 256, 0, st>>>(functional, p0, nvalid, ld, w, pt, tq, ld, partial);
  else k_functional_mgga<2><<<nb, 256, 0, st>>>(functional, p0, nvalid, ld, w, pt, tq, ld, partial);
  launch_sum_partials(partial, (int)nb, acc, st);
}

}  // namespace pgxc
