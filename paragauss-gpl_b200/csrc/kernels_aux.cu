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
// point).  So each P_i is formed here independently as that same ordered
// product, with the reference's rounding, and w = P_a / sum_i P_i with the sum
// in ascending i.
//
// Cost: natm^2 pair evaluations per point in the reference.  The kernel drops
// the terms that cannot matter at double precision:
//  * the nearest atom's P_near is formed first (exactly); sum_i P_i >= P_near;
//  * every factor is at most 1, so an atom whose product (or the product of
//    its factors with the four atoms nearest to the point) falls below
//    tau = 2^-56 P_near / natm contributes less than 2^-56 of the sum in
//    total: it is dropped (and w = 0 if it is the host atom).  The weights
//    then agree with the full ordered products to within 2^-56 relative (a
//    quarter of an ulp of the sum), and bit for bit at nearly every point;
//  * where mu <= -0.994 the rounded p3(mu) is -1 or -1 + 2^-53 and
//    s = (1 - p3)/2 rounds to exactly 1, so the factor leaves P unchanged and
//    is not evaluated (for x in [0.994, 1] the second iterate of p is
//    1 - e with e < 2^-27, and the third rounds to 1 or 1 - 2^-53).
// mu = d / R is the correctly rounded quotient by Markstein's method
// (P. W. Markstein, IBM J. Res. Dev. 34 (1990) 111): with y = RN(1/R),
// q = RN(d y), r = d - R q (exact with one FMA), mu = RN(q + r y).
// The point-atom distances are kept in shared memory (exact) for up to
// kBeckeCacheAtoms atoms and recomputed beyond.
// ---------------------------------------------------------------------------
// Arithmetic is written with explicit round-to-nearest intrinsics: no FMA
// contraction where the reference has none, so the factors round as the
// reference's IEEE double arithmetic.
__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// dist[i][j] = |R_i - R_j|; rdist[i][j] = RN(1 / dist[i][j]) (0 on the diagonal)
__global__ void k_atom_dist(const double* __restrict__ atoms, int natm, double* __restrict__ dist,
                            double* __restrict__ rdist) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= natm * natm) return;
  const int i = idx / natm, j = idx % natm;
  const int lo = i < j ? i : j, hi = i < j ? j : i;  // dst(lo,hi) computed once, mirrored
  const double d = dist3(atoms[3 * lo], atoms[3 * lo + 1], atoms[3 * lo + 2], atoms[3 * hi], atoms[3 * hi + 1],
                         atoms[3 * hi + 2]);
  dist[idx] = d;
  if (rdist) rdist[idx] = i == j ? 0.0 : __drcp_rn(d);
}

namespace {

constexpr int kBeckeThreads = 128;
constexpr int kBeckeCacheAtoms = 64;       // exact distance cache in shared memory up to this many atoms
constexpr double kBeckeEdge = 0.9941;      // d <= -kBeckeEdge R_ik => mu <= -0.994 after rounding

// d / R correctly rounded, y = RN(1 / R) (Markstein)
__device__ __forceinline__ double div_rn(double d, double R, double y) {
  const double q = __dmul_rn(d, y);
  const double r = __fma_rn(-q, R, d);
  return __fma_rn(r, y, q);
}

// s(mu_ik) of the reference for d = r_i - r_k and R = |R_i - R_k|.  The
// reference's pair orientation, mu = (r_i - r_k)/dst(k,i) for k < i and
// -(r_k - r_i)/dst(i,k) for k > i, is the same rounded value: IEEE
// subtraction and division are exactly antisymmetric.  mu0(mu, 0) =
// p(p(p(mu))), p(q) = q (3 - q^2) / 2; the halvings are multiplications by
// 0.5, which round exactly as the divisions by 2 do.
__device__ __forceinline__ double becke_s(double d, double R, double y) {
  double q = div_rn(d, R, y);
#pragma unroll
  for (int it = 0; it < 3; ++it) q = __dmul_rn(__dmul_rn(q, __dsub_rn(3.0, __dmul_rn(q, q))), 0.5);
  return __dmul_rn(__dsub_rn(1.0, q), 0.5);
}

template <bool kCache>
__global__ void __launch_bounds__(kBeckeThreads) k_becke(const double* __restrict__ atoms,
                                                         const double* __restrict__ dist,
                                                         const double* __restrict__ rdist, int natm,
                                                         const double* __restrict__ px, const double* __restrict__ py,
                                                         const double* __restrict__ pz,
                                                         const int* __restrict__ owner, int64_t n,
                                                         double* __restrict__ w) {
  extern __shared__ double sr[];  // kCache: r[k][thread]
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double x = px[p], y = py[p], z = pz[p];
  const int a = owner[p];
  auto r_of = [&](int k) {
    if (kCache) return sr[k * kBeckeThreads + threadIdx.x];
    return dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), x, y, z);
  };
  // the four atoms nearest to the point (sorted) and their distances
  int nb[4] = {-1, -1, -1, -1};
  double nr[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  for (int k = 0; k < natm; ++k) {
    const double r = dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), x, y, z);
    if (kCache) sr[k * kBeckeThreads + threadIdx.x] = r;
    if (r < nr[3]) {
      int j = 3;
      for (; j > 0 && nr[j - 1] > r; --j) {
        nr[j] = nr[j - 1];
        nb[j] = nb[j - 1];
      }
      nr[j] = r;
      nb[j] = k;
    }
  }
  // P_i as the ordered product, factors that are exactly 1 skipped; 0 once
  // the partial product is below tau (the factors left are at most 1)
  auto ordered = [&](int i, double ri, double tau) {
    const double* Ri = dist + (int64_t)i * natm;
    const double* Yi = rdist + (int64_t)i * natm;
    double P = 1.0;
    for (int k = 0; k < natm; ++k) {
      if (k == i) continue;
      const double R = __ldg(Ri + k);
      const double d = __dsub_rn(ri, r_of(k));
      if (d <= -__dmul_rn(kBeckeEdge, R)) continue;
      P = __dmul_rn(P, becke_s(d, R, __ldg(Yi + k)));
      if (P < tau) return 0.0;
    }
    return P;
  };
  const int i0 = nb[0];
  const double P0 = ordered(i0, nr[0], 0.0);
  const double tau = fmax(0x1p-56 * P0 / natm, 0x1p-1000);
  double sum = 0.0, pa = 0.0;
  for (int i = 0; i < natm; ++i) {
    double P;
    if (i == i0) {
      P = P0;
    } else {
      const double ri = r_of(i);
      const double* Ri = dist + (int64_t)i * natm;
      const double* Yi = rdist + (int64_t)i * natm;
      // bound from the nearest atoms
      double Q = 1.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int k = nb[c];
        if (k < 0 || k == i) continue;
        const double R = __ldg(Ri + k);
        const double d = __dsub_rn(ri, nr[c]);
        if (d > -__dmul_rn(kBeckeEdge, R)) Q *= becke_s(d, R, __ldg(Yi + k));
      }
      P = Q < tau ? 0.0 : ordered(i, ri, tau);
    }
    if (P != 0.0) sum = __dadd_rn(sum, P);  // zeros leave the ascending sum unchanged
    if (i == a) pa = P;
  }
  w[p] = __ddiv_rn(pa, sum);
}

}  // namespace

cudaError_t launch_becke(const double* atoms, double* dist, int natm, const double* px, const double* py,
                         const double* pz, const int* owner, int64_t n, double* w, cudaStream_t st) {
  // dist holds 2 natm^2 doubles: the distances, then their reciprocals
  double* rdist = dist + (int64_t)natm * natm;
  k_atom_dist<<<(natm * natm + 255) / 256, 256, 0, st>>>(atoms, natm, dist, rdist);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || n == 0) return e;
  const unsigned nb = (unsigned)((n + kBeckeThreads - 1) / kBeckeThreads);
  if (natm <= kBeckeCacheAtoms) {
    const int smem = natm * kBeckeThreads * (int)sizeof(double);
    e = cudaFuncSetAttribute(k_becke<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_becke<true><<<nb, kBeckeThreads, smem, st>>>(atoms, dist, rdist, natm, px, py, pz, owner, n, w);
  } else {
    k_becke<false><<<nb, kBeckeThreads, 0, st>>>(atoms, dist, rdist, natm, px, py, pz, owner, n, w);
  }
  return cudaGetLastError();
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
