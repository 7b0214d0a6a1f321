// kernels_aux.cu -- Becke partition weights and the point-wise functional.
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"
#include "xc_functional.cuh"

namespace pgxc {

// ---------------------------------------------------------------------------
// K0: Becke weights (becke0, modules/grid_module.f90:2442-2497; mu0 of
// autodiff/becke_step_func.f90:84-124 with art = 0).
//
// The reference accumulates P_i *= s_ik, P_k *= s_ki over pairs k < i.  For a
// fixed atom a this multiplies P_a by s_ak for the other atoms in ascending
// order, and s_ki = (1 - p3(mu_ki))/2 because p3 is odd (exactly, in floating
// point).  So each P_a is formed here independently as that same ordered
// product, giving the reference's rounding.  Once a product reaches exactly 0
// (s rounds to 0 when |mu| is close to 1) the remaining factors cannot change
// it and are skipped: the skip is exact.
// ---------------------------------------------------------------------------
// Arithmetic is written with explicit round-to-nearest intrinsics: no FMA
// contraction, so every weight is bit-identical to the reference's IEEE
// double arithmetic (which has no fused operations on its path).
__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

__global__ void k_atom_dist(const double* __restrict__ atoms, int natm, double* __restrict__ dist) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= natm * natm) return;
  const int i = idx / natm, j = idx % natm;
  const int lo = i < j ? i : j, hi = i < j ? j : i;  // dst(lo,hi) computed once, mirrored
  dist[idx] = dist3(atoms[3 * lo], atoms[3 * lo + 1], atoms[3 * lo + 2], atoms[3 * hi], atoms[3 * hi + 1],
                    atoms[3 * hi + 2]);
}

__global__ void __launch_bounds__(128) k_becke(const double* __restrict__ atoms, const double* __restrict__ dist,
                                               int natm, const double* __restrict__ px, const double* __restrict__ py,
                                               const double* __restrict__ pz, const int* __restrict__ owner,
                                               int64_t n, double* __restrict__ w) {
  extern __shared__ double sa[];  // natm * 3 coordinates
  for (int i = threadIdx.x; i < 3 * natm; i += blockDim.x) sa[i] = atoms[i];
  __syncthreads();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double x = px[p], y = py[p], z = pz[p];
  const int a = owner[p];
  double sum = 0.0, pa = 0.0;
  for (int i = 0; i < natm; ++i) {
    const double ri = dist3(sa[3 * i], sa[3 * i + 1], sa[3 * i + 2], x, y, z);
    double P = 1.0;
    for (int k = 0; k < natm && P != 0.0; ++k) {
      if (k == i) continue;
      const double rk = dist3(sa[3 * k], sa[3 * k + 1], sa[3 * k + 2], x, y, z);
      // the reference's pair orientation: mu = (r_i - r_k)/dst(k,i) for k < i
      double mu;
      if (k < i) mu = __ddiv_rn(__dsub_rn(ri, rk), __ldg(dist + k * natm + i));
      else mu = -__ddiv_rn(__dsub_rn(rk, ri), __ldg(dist + i * natm + k));
      // mu0(mu, 0) = p(p(p(mu))), p(q) = q (3 - q^2) / 2; the halvings are
      // multiplications by 0.5, which round exactly as the divisions by 2 do
      double q = mu;
#pragma unroll
      for (int it = 0; it < 3; ++it) q = __dmul_rn(__dmul_rn(q, __dsub_rn(3.0, __dmul_rn(q, q))), 0.5);
      P = __dmul_rn(P, __dmul_rn(__dsub_rn(1.0, q), 0.5));
    }
    sum = __dadd_rn(sum, P);
    if (i == a) pa = P;
  }
  w[p] = __ddiv_rn(pa, sum);
}

void launch_becke(const double* atoms, double* dist, int natm, const double* px, const double* py, const double* pz,
                  const int* owner, int64_t n, double* w, cudaStream_t st) {
  k_atom_dist<<<(natm * natm + 255) / 256, 256, 0, st>>>(atoms, natm, dist);
  const size_t smem = (size_t)(3 * natm) * sizeof(double);
  k_becke<<<(unsigned)((n + 127) / 128), 128, smem, st>>>(atoms, dist, natm, px, py, pz, owner, n, w);
}

__global__ void k_scale_inplace(double* __restrict__ x, const double* __restrict__ s, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s[i];
}

void launch_scale_inplace(double* x, const double* s, int64_t n, cudaStream_t st) {
  k_scale_inplace<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, s, n);
}

// ---------------------------------------------------------------------------
// xc_functionals on n points, closed shell.
// ---------------------------------------------------------------------------
__global__ void k_xc_points(XcConst K, int functional, int64_t n, const double* __restrict__ rho, const double* __restrict__ gam,
                            double* __restrict__ f, double* __restrict__ fr, double* __restrict__ fg) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (PGXC_XC_IS_GGA(functional)) {
    double a, b, c;
    xc_gga(K, rho[p], gam[p], a, b, c);
    f[p] = a; fr[p] = b; fg[p] = c;
  } else {
    double a, b;
    xc_vwn(K, rho[p], a, b);
    f[p] = a; fr[p] = b;
  }
}

// open shell: rho (n, 2), gam (n, 3) = (aa, bb, ab), fr (n, 2), fg (n, 3), column-major
template <bool GGA>
__global__ void k_xc_points2(XcConst K, int64_t n, const double* __restrict__ rho, const double* __restrict__ gam,
                             double* __restrict__ f, double* __restrict__ fr, double* __restrict__ fg) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double r[2] = {rho[p], rho[p + n]};
  const double g[3] = {GGA ? gam[p] : 0.0, GGA ? gam[p + n] : 0.0, GGA ? gam[p + 2 * n] : 0.0};
  double F, Fr[2], Fg[3];
  xc_open<GGA>(K, r, g, F, Fr, Fg);
  f[p] = F;
  fr[p] = Fr[0];
  fr[p + n] = Fr[1];
  if (GGA) {
    fg[p] = Fg[0];
    fg[p + n] = Fg[1];
    fg[p + 2 * n] = Fg[2];
  }
}

void launch_xc_points(int functional, int ispin, int64_t n, const double* rho, const double* gam, double* f,
                      double* fr, double* fg, cudaStream_t st) {
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (ispin == 1)
    k_xc_points<<<nb, 256, 0, st>>>(make_xc_const(functional), functional, n, rho, gam, f, fr, fg);
  else if (PGXC_XC_IS_GGA(functional))
    k_xc_points2<true><<<nb, 256, 0, st>>>(make_xc_const(functional), n, rho, gam, f, fr, fg);
  else
    k_xc_points2<false><<<nb, 256, 0, st>>>(make_xc_const(functional), n, rho, gam, f, fr, fg);
}

}  // namespace pgxc
