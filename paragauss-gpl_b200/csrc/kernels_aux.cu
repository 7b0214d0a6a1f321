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
//    its factors with the eight atoms nearest to the point) falls below
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
// p(p(p(mu))), p(q) = q (3 - q^2) / 2, s = (1 - q) / 2.  Halving is exact
// and commutes with rounding (no operand here is subnormal: |mu| is at least
// an ulp of a distance over a distance), so the reference's
// RN(RN(q RN(3 - RN(q q))) / 2) is RN(q RN(1.5 - RN(q q) / 2)), the inner
// step one FMA, and RN(1 - q) / 2 is the FMA RN(0.5 - q / 2): the same
// bits in 13 operations instead of 17.
__device__ __forceinline__ double becke_s(double d, double R, double y) {
  double q = div_rn(d, R, y);
#pragma unroll
  for (int it = 0; it < 3; ++it) q = __dmul_rn(q, __fma_rn(-0.5, __dmul_rn(q, q), 1.5));
  return __fma_rn(-0.5, q, 0.5);
}

// P_i = the ordered product over k != i of s(mu_ik) for the point whose
// distance to atom k is rk(k) (ri = rk(i)); 0 once the partial product is
// below tau.  Four factors are formed independently per step (their FP64
// chains overlap) and multiplied into P in ascending k; a factor that is
// skipped (k = i, or exactly 1) enters as 1.0, which leaves P bit for bit
// unchanged.  Every factor lies in [0, 1], so P never rises: testing tau once
// per step returns 0 exactly where the test after every factor would.
constexpr int kBeckeStep = 4;
template <class RK>
__device__ __forceinline__ double becke_product(int i, double ri, int natm, const double* __restrict__ Ri,
                                                const double* __restrict__ Yi, double tau, RK rk) {
  double P = 1.0;
  for (int k0 = 0; k0 < natm; k0 += kBeckeStep) {
    double f[kBeckeStep];
#pragma unroll
    for (int u = 0; u < kBeckeStep; ++u) {
      const int k = min(k0 + u, natm - 1);
      const double R = __ldg(Ri + k);
      const double d = __dsub_rn(ri, rk(k));
      const bool use = k0 + u < natm && k != i && d > -__dmul_rn(kBeckeEdge, R);
      f[u] = use ? becke_s(d, R, __ldg(Yi + k)) : 1.0;
    }
#pragma unroll
    for (int u = 0; u < kBeckeStep; ++u) P = __dmul_rn(P, f[u]);
    if (P < tau) return 0.0;
  }
  return P;
}

// The kNear atoms nearest to the point, kept sorted by distance (ties in
// ascending atom order): insert atom k at distance r.
constexpr int kNear = 8;
__device__ __forceinline__ void near_insert(int (&nb)[kNear], double (&nr)[kNear], int k, double r) {
  if (!(r < nr[kNear - 1])) return;
  int kk = k;
  double rr = r;
#pragma unroll
  for (int c = 0; c < kNear; ++c) {  // one pass of swaps keeps the array sorted
    if (rr < nr[c]) {
      const double tr = nr[c];
      const int tk = nb[c];
      nr[c] = rr;
      nb[c] = kk;
      rr = tr;
      kk = tk;
    }
  }
}
// Whether P_i can reach tau: every factor is at most 1, so P_i is at most the
// product of its factors with the nearest atoms; they are multiplied nearest
// first, which brings a far atom's bound below tau after a factor or two.
__device__ __forceinline__ bool near_bound(int i, double ri, const int (&nb)[kNear], const double (&nr)[kNear],
                                           const double* __restrict__ Ri, const double* __restrict__ Yi,
                                           double tau) {
  double Q = 1.0;
#pragma unroll
  for (int c = 0; c < kNear; ++c) {
    const int k = nb[c];
    if (k < 0 || k == i) continue;
    const double R = __ldg(Ri + k);
    const double d = __dsub_rn(ri, nr[c]);
    if (d > -__dmul_rn(kBeckeEdge, R)) Q *= becke_s(d, R, __ldg(Yi + k));
    if (Q < tau) return false;
  }
  return true;
}

// Thread per point (geometries of more than kBeckeWarpAtoms atoms).
__global__ void __launch_bounds__(kBeckeThreads) k_becke_thread(const double* __restrict__ atoms,
                                                                const double* __restrict__ dist,
                                                                const double* __restrict__ rdist, int natm,
                                                                const double* __restrict__ px,
                                                                const double* __restrict__ py,
                                                                const double* __restrict__ pz,
                                                                const int* __restrict__ owner, int64_t n,
                                                                double* __restrict__ w) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double x = px[p], y = py[p], z = pz[p];
  const int a = owner[p];
  auto r_of = [&](int k) {
    return dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), x, y, z);
  };
  // the kNear atoms nearest to the point (sorted) and their distances
  int nb[kNear];
  double nr[kNear];
#pragma unroll
  for (int c = 0; c < kNear; ++c) {
    nb[c] = -1;
    nr[c] = INFINITY;
  }
  for (int k = 0; k < natm; ++k) near_insert(nb, nr, k, r_of(k));
  // P_i as the ordered product, factors that are exactly 1 skipped; 0 once
  // the partial product is below tau (the factors left are at most 1)
  auto ordered = [&](int i, double ri, double tau) {
    return becke_product(i, ri, natm, dist + (int64_t)i * natm, rdist + (int64_t)i * natm, tau, r_of);
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
      // bound from the nearest atoms
      P = near_bound(i, ri, nb, nr, dist + (int64_t)i * natm, rdist + (int64_t)i * natm, tau) ? ordered(i, ri, tau)
                                                                                             : 0.0;
    }
    if (P != 0.0) sum = __dadd_rn(sum, P);  // zeros leave the ascending sum unchanged
    if (i == a) pa = P;
  }
  w[p] = __ddiv_rn(pa, sum);
}

// The same weights with the surviving (point, atom) products spread over the
// lanes of a warp (for up to kBeckeWarpAtoms atoms).  Thread per point, each
// lane first finds its point's nearest atoms, the nearest atom's P, tau and a
// bitmask of the atoms whose bound Q_i reaches tau; the warp then computes the
// ordered products of all its points' surviving atoms 32 at a time (lane l
// takes the l-th pending pair, whatever point it belongs to), and each
// product is handed back to its point's lane in ascending atom order, so
// every point's sum is formed in the reference's order.  Thread-per-point
// loops over the atoms diverge wherever the lanes' points keep different
// atoms; here every lane of a round has a product to form.
//
// The survivor bitmasks live in shared memory, word u of lane l at
// [u][l] of the warp's block (ceil(natm / 32) words per point).
//
// A round's 32 pairs belong to few points (2.8 on average at 60 atoms), and
// each ordered product needs the point's distance to every atom.  Up to
// kTabAtoms atoms the warp therefore first writes the distances of the
// round's first kTabPts points to all atoms into a shared table (the same
// correctly rounded dist3 values) and the products read them there; a lane
// whose point is not in the table (a round of more than kTabPts points), and
// every lane beyond kTabAtoms atoms, computes its distances itself.
constexpr int kBeckeWarpAtoms = 1024;
constexpr int kTabAtoms = 256;
constexpr int kTabPts = 4;

// dynamic shared memory of one warp: the masks, then the distance table
__host__ __device__ constexpr int becke_warp_smem(int natm) {
  return 128 * ((natm + 31) / 32) + (natm <= kTabAtoms ? kTabPts * natm * 8 : 0);
}

__global__ void __launch_bounds__(kBeckeThreads) k_becke_warp(const double* __restrict__ atoms,
                                                              const double* __restrict__ dist,
                                                              const double* __restrict__ rdist, int natm,
                                                              const double* __restrict__ px,
                                                              const double* __restrict__ py,
                                                              const double* __restrict__ pz,
                                                              const int* __restrict__ owner, int64_t n,
                                                              double* __restrict__ w) {
  extern __shared__ double becke_sm[];
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int mw = (natm + 31) / 32;
  unsigned* wmask = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(becke_sm) +
                                                (threadIdx.x >> 5) * becke_warp_smem(natm));
  double* tab = reinterpret_cast<double*>(wmask + 32 * mw);  // natm <= kTabAtoms only
  const bool use_tab = natm <= kTabAtoms;
  const bool live = p < n;  // every lane takes part in the warp's rounds
  double x = 0.0, y = 0.0, z = 0.0;
  int a = -1;
  if (live) {
    x = px[p];
    y = py[p];
    z = pz[p];
    a = owner[p];
  }
  // P_i of the point at (qx, qy, qz): the ordered product, exactly-1 factors
  // skipped, 0 once below tau
  auto ordered = [&](int i, double qx, double qy, double qz, double tau) {
    auto rk = [&](int k) {
      return dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), qx, qy, qz);
    };
    return becke_product(i, rk(i), natm, dist + (int64_t)i * natm, rdist + (int64_t)i * natm, tau, rk);
  };
  // the same product with the point's distances to the atoms read from rt
  auto ordered_tab = [&](int i, const double* rt, double tau) {
    return becke_product(i, rt[i], natm, dist + (int64_t)i * natm, rdist + (int64_t)i * natm, tau,
                         [&](int k) { return rt[k]; });
  };
  int nb[kNear];
  double nr[kNear];
#pragma unroll
  for (int c = 0; c < kNear; ++c) {
    nb[c] = -1;
    nr[c] = INFINITY;
  }
  int cnt = 0;
  double P0 = 0.0, tau = 0.0;
  int i0 = -1;
  if (live) {
    for (int k = 0; k < natm; ++k) {
      const double r = dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), x, y, z);
      near_insert(nb, nr, k, r);
    }
    i0 = nb[0];
    P0 = ordered(i0, x, y, z, 0.0);
    tau = fmax(0x1p-56 * P0 / natm, 0x1p-1000);
    unsigned word = 0;
    for (int i = 0; i < natm; ++i) {
      if ((i & 31) == 0 && i > 0) {
        wmask[32 * ((i >> 5) - 1) + lane] = word;
        word = 0;
      }
      if (i == i0) continue;
      const double ri = dist3(__ldg(atoms + 3 * i), __ldg(atoms + 3 * i + 1), __ldg(atoms + 3 * i + 2), x, y, z);
      if (near_bound(i, ri, nb, nr, dist + (int64_t)i * natm, rdist + (int64_t)i * natm, tau)) {
        word |= 1u << (i & 31);
        ++cnt;
      }
    }
    wmask[32 * (mw - 1) + lane] = word;
  } else {
    for (int u = 0; u < mw; ++u) wmask[32 * u + lane] = 0u;
  }
  __syncwarp();
  // the warp's pending pairs: lane l's are positions off .. off + cnt - 1, ascending atom
  int off = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, off, d);
    if (lane >= d) off += v;
  }
  const int total = __shfl_sync(0xffffffffu, off, 31);
  off -= cnt;
  double sum = 0.0, pa = 0.0;
  bool p0_added = false;
  auto add = [&](int i, double P) {  // this lane's point: the next product in ascending atom order
    if (!p0_added && i > i0) {
      if (P0 != 0.0) sum = __dadd_rn(sum, P0);
      if (a == i0) pa = P0;
      p0_added = true;
    }
    if (P != 0.0) sum = __dadd_rn(sum, P);
    if (i == a) pa = P;
  };
  for (int base = 0; base < total; base += 32) {
    const int q = base + lane;
    // owner lane of position q: the largest l with off_l <= q
    int ol = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
      const int cand = ol + st;
      const int oc = __shfl_sync(0xffffffffu, off, cand & 31);
      if (cand < 32 && oc <= q) ol = cand;
    }
    const int j = q - __shfl_sync(0xffffffffu, off, ol);  // rank of the pair among the owner's
    const double qx = __shfl_sync(0xffffffffu, x, ol), qy = __shfl_sync(0xffffffffu, y, ol),
                 qz = __shfl_sync(0xffffffffu, z, ol), qt = __shfl_sync(0xffffffffu, tau, ol);
    // the round's points in lane order (owners ascend with the position);
    // jd = this lane's point among them
    const int olp = __shfl_up_sync(0xffffffffu, ol, 1);
    const unsigned fm = __ballot_sync(0xffffffffu, q < total && (lane == 0 || olp != ol));
    const int jd = __popc(fm & ((2u << lane) - 1u)) - 1;
    const int md = use_tab ? min(__popc(fm), kTabPts) : 0;
    __syncwarp();  // the previous round's reads of the table are done
    for (int jt = 0; jt < md; ++jt) {
      const int src = __shfl_sync(0xffffffffu, ol, (int)__fns(fm, 0, jt + 1));
      const double tx = __shfl_sync(0xffffffffu, x, src), ty = __shfl_sync(0xffffffffu, y, src),
                   tz = __shfl_sync(0xffffffffu, z, src);
      for (int k = lane; k < natm; k += 32)
        tab[jt * natm + k] = dist3(__ldg(atoms + 3 * k), __ldg(atoms + 3 * k + 1), __ldg(atoms + 3 * k + 2), tx, ty, tz);
    }
    __syncwarp();
    int pi = -1;
    double P = 0.0;
    if (q < total) {
      int r = j;
      for (int u = 0; u < mw; ++u) {
        const unsigned mu = wmask[32 * u + ol];
        const int c = __popc(mu);
        if (r < c) {
          pi = 32 * u + (int)__fns(mu, 0, r + 1);
          break;
        }
        r -= c;
      }
      P = jd < md ? ordered_tab(pi, tab + jd * natm, qt) : ordered(pi, qx, qy, qz, qt);
    }
    // hand the round's products to their points' lanes, in position order
    for (int t = 0; t < 32; ++t) {
      const int tl = __shfl_sync(0xffffffffu, ol, t), ti = __shfl_sync(0xffffffffu, pi, t);
      const double tp = __shfl_sync(0xffffffffu, P, t);
      if (base + t < total && tl == lane) add(ti, tp);
    }
  }
  if (live) {
    if (!p0_added) {
      if (P0 != 0.0) sum = __dadd_rn(sum, P0);
      if (a == i0) pa = P0;
    }
    w[p] = __ddiv_rn(pa, sum);
  }
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
  if (natm <= kBeckeWarpAtoms)
    k_becke_warp<<<nb, kBeckeThreads, (kBeckeThreads / 32) * becke_warp_smem(natm), st>>>(
        atoms, dist, rdist, natm, px, py, pz, owner, n, w);
  else
    k_becke_thread<<<nb, kBeckeThreads, 0, st>>>(atoms, dist, rdist, natm, px, py, pz, owner, n, w);
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
