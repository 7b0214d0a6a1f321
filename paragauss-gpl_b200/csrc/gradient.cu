// gradient.cu -- kernels of the post-SCF XC nuclear gradient (gradient.h).
//
// FP64 throughout.  The gradient runs once per geometry, after the SCF: the
// kernels are plain per-point / per-function loops; the four contractions
// per spin (X = Phi P, Y_j = d_j Phi P) are library DGEMMs issued by the caller.
#include <cmath>

#include "basis.cuh"
#include "dgemm.cuh"
#include "gradient.h"
#include "xc_functional.cuh"
#include "xc_mgga.cuh"

namespace pgxc {

namespace {

// Real solid harmonics, first and second derivatives, by the recursion of
// solid_harmonics (basis.cuh, modules/solid_harmonics_module.f90:369-482)
// differentiated twice.  H[k][.] holds xx, xy, xz, yy, yz, zz.
template <int L>
__device__ __forceinline__ void solid_harmonics_h(double x, double y, double z, double* Y, double (*dY)[16],
                                                  double (*H)[16]) {
  const double r2 = x * x + y * y + z * z;
  const double xv[3] = {x, y, z};
  constexpr int ci[6] = {0, 0, 0, 1, 1, 2}, di[6] = {0, 1, 2, 1, 2, 2};
  for (int i = 0; i < 16; ++i) {
    Y[i] = 0.0;
    for (int c = 0; c < 3; ++c) dY[c][i] = 0.0;
    for (int k = 0; k < 6; ++k) H[k][i] = 0.0;
  }
  Y[0] = 1.0;
  if (L == 0) return;
  Y[1] = z; Y[2] = x; Y[3] = y;
  dY[2][1] = 1.0; dY[0][2] = 1.0; dY[1][3] = 1.0;
#pragma unroll
  for (int l = 2; l <= L; ++l) {
    const int o = l * l, o1 = (l - 1) * (l - 1), o2 = (l - 2) * (l - 2);
    const double lr = l, l1r = l - 1, ll1r = 2 * l - 1;
    {
      const double p1 = Y[o1], p2 = Y[o2];
      Y[o] = (ll1r * z * p1 - l1r * r2 * p2) / lr;
      for (int c = 0; c < 3; ++c)
        dY[c][o] = (ll1r * ((c == 2 ? p1 : 0.0) + z * dY[c][o1]) - l1r * (2.0 * xv[c] * p2 + r2 * dY[c][o2])) / lr;
      for (int k = 0; k < 6; ++k) {
        const int c = ci[k], d = di[k];
        const double t1 = (c == 2 ? dY[d][o1] : 0.0) + (d == 2 ? dY[c][o1] : 0.0) + z * H[k][o1];
        const double t2 = (c == d ? 2.0 * p2 : 0.0) + 2.0 * xv[c] * dY[d][o2] + 2.0 * xv[d] * dY[c][o2] + r2 * H[k][o2];
        H[k][o] = (ll1r * t1 - l1r * t2) / lr;
      }
    }
    for (int im = 1; im <= l - 2; ++im) {
      const double sim = im * im;
      const double rlm = 1.0 / sqrt(lr * lr - sim);
      const double rl1m = sqrt(l1r * l1r - sim);
      const double a = ll1r * z * rlm;
      const double b = rl1m * r2 * rlm;
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const double p1 = Y[o1 + mm], p2 = Y[o2 + mm];
        Y[o + mm] = a * p1 - b * p2;
        for (int c = 0; c < 3; ++c)
          dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : 0.0) + a * dY[c][o1 + mm] - rl1m * 2.0 * xv[c] * rlm * p2 -
                          b * dY[c][o2 + mm];
        for (int k = 0; k < 6; ++k) {
          const int c = ci[k], d = di[k];
          H[k][o + mm] = (c == 2 ? ll1r * rlm * dY[d][o1 + mm] : 0.0) + (d == 2 ? ll1r * rlm * dY[c][o1 + mm] : 0.0) +
                         a * H[k][o1 + mm] -
                         rl1m * rlm * ((c == d ? 2.0 * p2 : 0.0) + 2.0 * xv[c] * dY[d][o2 + mm] + 2.0 * xv[d] * dY[c][o2 + mm]) -
                         b * H[k][o2 + mm];
        }
      }
    }
    {
      const int im = l - 1;
      const double rlm = 1.0 / sqrt(lr * lr - (double)(im * im));
      const double a = ll1r * z * rlm;
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const double p1 = Y[o1 + mm];
        Y[o + mm] = a * p1;
        for (int c = 0; c < 3; ++c) dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : 0.0) + a * dY[c][o1 + mm];
        for (int k = 0; k < 6; ++k) {
          const int c = ci[k], d = di[k];
          H[k][o + mm] = (c == 2 ? ll1r * rlm * dY[d][o1 + mm] : 0.0) + (d == 2 ? ll1r * rlm * dY[c][o1 + mm] : 0.0) +
                         a * H[k][o1 + mm];
        }
      }
    }
    {
      const double rll = sqrt(ll1r / (2.0 * lr));
      const int j2 = o1 + 2 * l - 3, j1 = o1 + 2 * l - 2;
      const double q2 = Y[j2], q1 = Y[j1];
      Y[o + 2 * l - 1] = (x * q2 - y * q1) * rll;
      Y[o + 2 * l] = (y * q2 + x * q1) * rll;
      for (int c = 0; c < 3; ++c) {
        const double dx = c == 0, dy = c == 1;
        dY[c][o + 2 * l - 1] = (dx * q2 + x * dY[c][j2] - dy * q1 - y * dY[c][j1]) * rll;
        dY[c][o + 2 * l] = (dy * q2 + y * dY[c][j2] + dx * q1 + x * dY[c][j1]) * rll;
      }
      for (int k = 0; k < 6; ++k) {
        const int c = ci[k], d = di[k];
        const double cx = c == 0, cy = c == 1, dx = d == 0, dy = d == 1;
        H[k][o + 2 * l - 1] = (cx * dY[d][j2] + dx * dY[c][j2] + x * H[k][j2] - cy * dY[d][j1] - dy * dY[c][j1] -
                               y * H[k][j1]) * rll;
        H[k][o + 2 * l] = (cy * dY[d][j2] + dy * dY[c][j2] + y * H[k][j2] + cx * dY[d][j1] + dx * dY[c][j1] +
                           x * H[k][j1]) * rll;
      }
    }
  }
}

// grid = (ld / 128, shells of L): phi, grad and Hessian of every function of the shell
template <int L>
__global__ void __launch_bounds__(128) k_basis_hess(const DevShell* __restrict__ shells, const int* __restrict__ ids,
                                                    const double* __restrict__ atoms, const double* __restrict__ exps,
                                                    const double* __restrict__ norms, const double* __restrict__ contr,
                                                    const int2* __restrict__ rng, DevSA sa,
                                                    const double* __restrict__ px, const double* __restrict__ py,
                                                    const double* __restrict__ pz, int64_t p0, int64_t nvalid,
                                                    int64_t ld, int64_t plane, double* __restrict__ out) {
  const DevShell S = shells[ids[blockIdx.y]];
  const int64_t p = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (p >= ld) return;
  const bool valid = p < nvalid;
  double x = 0, y = 0, z = 0;
  if (valid) {
    x = px[p0 + p] - atoms[3 * S.atom];
    y = py[p0 + p] - atoms[3 * S.atom + 1];
    z = pz[p0 + p] - atoms[3 * S.atom + 2];
  }
  double Y[16], dY[3][16], H[6][16];
  solid_harmonics_h<L>(x, y, z, Y, dY, H);
  const double r2 = x * x + y * y + z * z;
  const double xv[3] = {x, y, z};
  constexpr int ci[6] = {0, 0, 0, 1, 1, 2}, di[6] = {0, 1, 2, 1, 2, 2};
  // symmetry-adapted harmonics of this l
  double Ys[2 * L + 1], dYs[3][2 * L + 1], Hs[6][2 * L + 1];
  for (int i = 0; i < 2 * L + 1; ++i) {
    double v = 0, g[3] = {0, 0, 0}, h[6] = {0, 0, 0, 0, 0, 0};
    for (int m = 0; m < 2 * L + 1; ++m) {
      const double cf = sa.identity ? (m == i ? 1.0 : 0.0) : sa.c[L][i][m];
      v += cf * Y[L * L + m];
      for (int c = 0; c < 3; ++c) g[c] += cf * dY[c][L * L + m];
      for (int k = 0; k < 6; ++k) h[k] += cf * H[k][L * L + m];
    }
    Ys[i] = v;
    for (int c = 0; c < 3; ++c) dYs[c][i] = g[c];
    for (int k = 0; k < 6; ++k) Hs[k][i] = h[k];
  }
  const double* ex = exps + S.exp_off;
  const double* nr = norms + S.exp_off;
  const double* cc = contr + S.con_off;
  for (int rr = 0; rr < S.nrad; ++rr) {
    // R, dR = sum c (-2 alpha) v and d2R = sum c (4 alpha^2) v of radial function rr:
    // d_c R = x_c dR, d_c d_d R = delta_cd dR + x_c x_d d2R
    double R = 0.0, dR = 0.0, d2R = 0.0;
    if (valid) {
      int e0 = 0, e1 = S.nexp;
      if (S.seg) {
        const int2 rg = rng[S.rad_off + rr];
        e0 = rg.x;
        e1 = rg.y;
      }
      for (int e = e0; e < e1; ++e) {
        double cf;
        if (S.seg) cf = cc[e + (int64_t)S.nexp * rr];
        else if (rr < S.nunc) cf = (e == rr) ? 1.0 : 0.0;
        else cf = cc[e + (int64_t)S.nexp * (rr - S.nunc)];
        const double alpha = ex[e];
        const double v = prim_value(alpha, nr[e], r2);
        R += cf * v;
        dR += cf * (-2.0 * alpha) * v;
        d2R += cf * (4.0 * alpha * alpha) * v;
      }
    }
    for (int i = 0; i < 2 * L + 1; ++i) {
      const int64_t f = S.f0 + (int64_t)i * S.nrad + rr;
      double* o = out + f * ld + p;
      o[0] = Ys[i] * R;
      for (int c = 0; c < 3; ++c) o[(1 + c) * plane] = dYs[c][i] * R + Ys[i] * xv[c] * dR;
      for (int k = 0; k < 6; ++k) {
        const int c = ci[k], d = di[k];
        o[(4 + k) * plane] = Hs[k][i] * R + (dYs[c][i] * xv[d] + dYs[d][i] * xv[c]) * dR +
                             Ys[i] * ((c == d ? dR : 0.0) + xv[c] * xv[d] * d2R);
      }
    }
  }
}

// index of the Hessian component (c, d) in xx, xy, xz, yy, yz, zz
__device__ __forceinline__ int hidx(int c, int d) {
  const int a = c < d ? c : d, b = c < d ? d : c;
  return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

// coef planes per spin: a, b_x, b_y, b_z, c (c = w df/dtau, meta-GGAs)
constexpr int kCoefPlanes = 5;

__global__ void k_grad_points(XcConst K, int functional, bool gga, int ispin, int64_t nbas, int64_t ld, int64_t p0,
                              int64_t nvalid, const double* __restrict__ w, const double* __restrict__ wraw,
                              const double* __restrict__ B, int64_t plane, const double* __restrict__ XY,
                              double* __restrict__ coef, double* __restrict__ ef, double* __restrict__ exc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ld) return;
  if (p >= nvalid) {
    for (int s = 0; s < ispin; ++s)
      for (int c = 0; c < kCoefPlanes; ++c) coef[(kCoefPlanes * s + c) * ld + p] = 0.0;
    ef[p] = 0.0;
    return;
  }
  const bool mgga = PGXC_XC_IS_MGGA(functional);
  // rho_s, grad rho_s and (meta-GGAs) tau_s = 1/2 sum_j d_j phi P_s d_j phi = 1/2 sum_j,f d_j phi_f Y_j,f
  double rho[2] = {0, 0}, gr[2][3] = {{0, 0, 0}, {0, 0, 0}}, tau[2] = {0, 0};
  for (int s = 0; s < ispin; ++s) {
    const double* X = XY + (4 * s) * plane;
    for (int64_t f = 0; f < nbas; ++f) {
      const double xv = X[f * ld + p];
      rho[s] += B[f * ld + p] * xv;
      if (gga)
        for (int c = 0; c < 3; ++c) gr[s][c] += 2.0 * B[(1 + c) * plane + f * ld + p] * xv;
      if (mgga)
        for (int c = 0; c < 3; ++c) tau[s] += 0.5 * B[(1 + c) * plane + f * ld + p] * X[(1 + c) * plane + f * ld + p];
    }
  }
  const double wp = w[p0 + p];
  double f = 0.0, fr[2] = {0, 0}, fg[3] = {0, 0, 0}, ft[2] = {0, 0};
  if (ispin == 1) {
    const double g = gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2];
    if (mgga) mgga::mgga_closed(functional, rho[0], g, tau[0], f, fr[0], fg[0], ft[0]);
    else if (gga) xc_gga(K, rho[0], g, f, fr[0], fg[0]);
    else xc_vwn(K, rho[0], f, fr[0]);
    coef[p] = wp * fr[0];
    for (int c = 0; c < 3; ++c) coef[(1 + c) * ld + p] = gga ? wp * 2.0 * fg[0] * gr[0][c] : 0.0;
    coef[4 * ld + p] = wp * ft[0];
  } else {
    const double r2[2] = {rho[0], rho[1]};
    const double g3[3] = {gr[0][0] * gr[0][0] + gr[0][1] * gr[0][1] + gr[0][2] * gr[0][2],
                          gr[1][0] * gr[1][0] + gr[1][1] * gr[1][1] + gr[1][2] * gr[1][2],
                          gr[0][0] * gr[1][0] + gr[0][1] * gr[1][1] + gr[0][2] * gr[1][2]};
    double fr2[2], fg3[3];
    if (mgga) mgga::mgga_open(functional, r2, g3, tau, f, fr2, fg3, ft);
    else if (gga) xc_open<true>(K, r2, g3, f, fr2, fg3);
    else xc_open<false>(K, r2, g3, f, fr2, fg3);
    for (int s = 0; s < 2; ++s) {
      coef[(kCoefPlanes * s) * ld + p] = wp * fr2[s];
      for (int c = 0; c < 3; ++c)
        coef[(kCoefPlanes * s + 1 + c) * ld + p] = gga ? wp * (2.0 * fg3[s] * gr[s][c] + fg3[2] * gr[1 - s][c]) : 0.0;
      coef[(kCoefPlanes * s + 4) * ld + p] = wp * ft[s];
    }
  }
  ef[p] = wraw[p0 + p] * f;
  atomicAdd(exc, wp * f);
}

// The orbital terms in one pass: q^s_mu,k(p) is formed once per function and
// point.  Block = 256 points x kGradFB functions: each thread takes one point
// and loops over the block's functions; -q goes to atom(mu) through a warp
// reduction and the block's shared sums, +q to the point's host through the
// thread's running sum, reduced over the warp when all its points share a
// host (the usual case: the raw grid is atom by atom) and the block's shared
// per-atom sums.
// GGAs (not meta-GGAs): the Y_j enter the orbital terms only as
// sum_j b_j Y_j = W P with W = sum_j b_j d_j phi, one product instead of
// three.  W[f][p] for f < nbas, and zero rows nbas .. kpad - 1 (read by the
// product's K loop, which meets P's zero rows there).
__global__ void k_grad_w(int64_t nbas, int64_t kpad, int64_t ld, const double* __restrict__ B, int64_t plane,
                         const double* __restrict__ cb, double* __restrict__ W) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kpad * ld) return;
  const int64_t f = i / ld, p = i - f * ld;
  double w = 0.0;
  if (f < nbas)
    for (int j = 0; j < 3; ++j) w += cb[j * ld + p] * B[(1 + j) * plane + i];
  W[i] = w;
}

constexpr int kGradFB = 32;

__global__ void __launch_bounds__(256) k_grad_orb(bool gga, bool mgga, int ispin, int64_t nbas, int64_t ld, int64_t p0,
                                                  int64_t nvalid, int natm, const int* __restrict__ fatom,
                                                  const int* __restrict__ owner, const double* __restrict__ B,
                                                  int64_t plane, const double* __restrict__ XY,
                                                  const double* __restrict__ coef, double* __restrict__ grad) {
  extern __shared__ double sh[];  // [kGradFB][3] function sums, then [natm][3] host sums
  double* gq = sh;
  double* gh = sh + 3 * kGradFB;
  for (int i = threadIdx.x; i < 3 * (kGradFB + natm); i += blockDim.x) sh[i] = 0.0;
  __syncthreads();
  const int64_t p = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
  const bool live = p < nvalid;
  const int lane = threadIdx.x & 31;
  const int64_t f0 = (int64_t)blockIdx.x * kGradFB, f1 = min(nbas, f0 + kGradFB);
  // the point's coefficients, once for all its functions
  double a[2] = {0, 0}, b[2][3] = {{0, 0, 0}, {0, 0, 0}}, ct[2] = {0, 0};
  if (live)
    for (int sp = 0; sp < ispin; ++sp) {
      a[sp] = coef[(kCoefPlanes * sp) * ld + p];
      if (gga)
        for (int j = 0; j < 3; ++j) b[sp][j] = coef[(kCoefPlanes * sp + 1 + j) * ld + p];
      if (mgga) ct[sp] = coef[(kCoefPlanes * sp + 4) * ld + p];
    }
  double t[3] = {0, 0, 0};
  for (int64_t f = f0; f < f1; ++f) {
    double q[3] = {0, 0, 0};
    if (live) {
      const int64_t o = f * ld + p;
      double d[3], H[6];
      for (int c = 0; c < 3; ++c) d[c] = B[(1 + c) * plane + o];
      if (gga)
        for (int k = 0; k < 6; ++k) H[k] = B[(4 + k) * plane + o];
      for (int sp = 0; sp < ispin; ++sp) {
        const double X = XY[(4 * sp) * plane + o];
        for (int k = 0; k < 3; ++k) q[k] += 2.0 * a[sp] * d[k] * X;
        if (!gga) continue;
        if (!mgga) {  // sum_j b_j Y_j = (sum_j b_j d_j phi) P = V, plane 2 of the spin
          const double V = XY[(4 * sp + 2) * plane + o];
          for (int k = 0; k < 3; ++k) {
            double u = d[k] * V;
            for (int j = 0; j < 3; ++j) u += b[sp][j] * H[hidx(k, j)] * X;
            q[k] += 2.0 * u;
          }
          continue;
        }
        double Yj[3];
        for (int j = 0; j < 3; ++j) Yj[j] = XY[(4 * sp + 1 + j) * plane + o];
        for (int k = 0; k < 3; ++k) {
          double u = 0.0;
          for (int j = 0; j < 3; ++j) u += b[sp][j] * (H[hidx(k, j)] * X + d[k] * Yj[j]);
          q[k] += 2.0 * u;
          // meta-GGAs: tau moves with the functions through d_k d_j phi
          if (mgga)
            for (int j = 0; j < 3; ++j) q[k] += ct[sp] * H[hidx(k, j)] * Yj[j];
        }
      }
    }
    for (int k = 0; k < 3; ++k) {
      t[k] += q[k];
      double v = q[k];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0 && v != 0.0) atomicAdd(&gq[3 * (f - f0) + k], v);
    }
  }
  // host sums: one shared atomic per warp when its points share a host
  const int h = live ? owner[p0 + p] : -1;
  const int h0 = __shfl_sync(0xffffffffu, h, 0);
  if (__all_sync(0xffffffffu, h == h0) && h0 >= 0) {
    for (int k = 0; k < 3; ++k) {
      double v = t[k];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) atomicAdd(&gh[3 * h0 + k], v);
    }
  } else if (live) {
    for (int k = 0; k < 3; ++k) atomicAdd(&gh[3 * h + k], t[k]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * (int)(f1 - f0); i += blockDim.x)
    if (gq[i] != 0.0) atomicAdd(grad + 3 * fatom[f0 + i / 3] + i % 3, -gq[i]);
  for (int i = threadIdx.x; i < 3 * natm; i += blockDim.x)
    if (gh[i] != 0.0) atomicAdd(grad + i, gh[i]);
}

// Thread per point.  Pass 1 stores, per atom b, the point's distance d_b,
// its reciprocal and the row of P_b = prod_{c != b} s(mu_bc): the product of
// its nonzero factors, their zero count and the index of a zero factor
// (scratch [atom][ld]).  Pass 2 gathers, per atom x, the terms of the pairs
// (x, y) and (y, x) in registers (no scatter):
//   dmu_xy/dR_x = -u_x/R - mu r_xy/R^2,  dmu_yx/dR_x = u_x/R + mu r_xy/R^2,
//   kappa_xy = c_x L_xy s'(mu_xy), c_b = ef (delta_bh - W_h) / Z,
// L_xy the product of row x without its factor y; the point moves with its
// host h, which collects kappa_xy (u_x - u_y)/R of every pair.  Each atom's sum
// is reduced over the warp and added to shared memory, then to grad.
//
// Rows whose leave-one-out products are all negligible ("dead" rows) take
// part only through their pairs with live rows.  Every factor is at most 1,
// so L_xy <= the product of row x's factors with the eight atoms nearest to the
// point, leaving out the smallest of them; where that bound is below 2^-60
// the row is dead (its P_x is below the same bound and is dropped from Z).
// Both loops of pass 2 run over all atoms in the same order on every lane of
// a warp; a pair is skipped when, for every lane, both its rows are dead.
// Where mu <= -0.994, s rounds to exactly 1 and leaves the row product
// unchanged.
//
// mu_bc = (d_b - d_c) RN(1/R_bc): pass 1 and pass 2 form it alike, and
// mu_cb = -mu_bc exactly, so s(mu_cb) = (1 + p3(mu_bc))/2 with the same
// bits as pass 1's factor (p3 is odd in floating point too): a factor that is
// exactly 0 in one pass is 0 in the other.
constexpr double kGradEdge = 0.9941;
constexpr double kGradTau = 0x1p-60;
constexpr int kGradNear = 8;  // atoms nearest to the point in the dead-row bound

// p3(mu) and ds/dmu (even in mu).  Each step RN(RN(q / 2) RN(3 - RN(q q)))
// is formed as RN(q RN(1.5 - RN(q q) / 2)) (one FMA inside): halving is exact
// and commutes with rounding for these normal operands, so the bits agree.
__device__ __forceinline__ void becke_p3(double mu, double& q3, double& ds) {
  const double q1 = __dmul_rn(mu, __fma_rn(-0.5, __dmul_rn(mu, mu), 1.5));
  const double q2 = __dmul_rn(q1, __fma_rn(-0.5, __dmul_rn(q1, q1), 1.5));
  q3 = __dmul_rn(q2, __fma_rn(-0.5, __dmul_rn(q2, q2), 1.5));
  ds = -0.5 * (1.5 * (1.0 - q2 * q2)) * (1.5 * (1.0 - q1 * q1)) * (1.5 * (1.0 - mu * mu));
}

template <bool MASK>
__global__ void __launch_bounds__(128) k_grad_weights(const double* __restrict__ atoms,
                                                      const double* __restrict__ dist,
                                                      const double* __restrict__ rdist, int natm,
                                                      const double* __restrict__ px, const double* __restrict__ py,
                                                      const double* __restrict__ pz, const int* __restrict__ owner,
                                                      int64_t p0, int64_t nvalid, int64_t ld,
                                                      const double* __restrict__ ef, double* __restrict__ sd,
                                                      double* __restrict__ sinv, double* __restrict__ spnz,
                                                      int* __restrict__ snz, double* __restrict__ grad) {
  extern __shared__ double G[];  // 3 natm sums of the block
  for (int i = threadIdx.x; i < 3 * natm; i += blockDim.x) G[i] = 0.0;
  __syncthreads();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < nvalid && ef[p] != 0.0;
  double rv[3] = {0, 0, 0}, e = 0.0, Z = 0.0, Wh = 0.0;
  int h = 0;
  uint64_t live_lo = 0, live_hi = 0;  // live rows of the point (atoms < 128; MASK)
  if (live) {
    rv[0] = px[p0 + p]; rv[1] = py[p0 + p]; rv[2] = pz[p0 + p];
    h = owner[p0 + p];
    e = ef[p];
    int nb[kGradNear];
    double nr[kGradNear];
#pragma unroll
    for (int c = 0; c < kGradNear; ++c) {
      nb[c] = -1;
      nr[c] = INFINITY;
    }
    for (int b = 0; b < natm; ++b) {
      const double t0 = rv[0] - atoms[3 * b], t1 = rv[1] - atoms[3 * b + 1], t2 = rv[2] - atoms[3 * b + 2];
      const double r = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
      sd[b * ld + p] = r;
      sinv[b * ld + p] = r > 0.0 ? 1.0 / r : 0.0;
      if (r < nr[kGradNear - 1]) {  // keep the kGradNear nearest sorted (ties in ascending atom order)
        int kk = b;
        double rr = r;
#pragma unroll
        for (int c = 0; c < kGradNear; ++c) {
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
    }
    double Ph = 0.0;
    for (int b = 0; b < natm; ++b) {
      const double db = sd[b * ld + p];
      const double* Rb = dist + (int64_t)b * natm;
      const double* Yb = rdist + (int64_t)b * natm;
      // bound: the near factors' product with its smallest factor left out (with
      // no zero factor Q / smin; with one, Q, the others; with more, 0).  Taking
      // in a further factor never raises it, so the nearest atoms come first and
      // the loop stops once it is below tau.
      double Q = 1.0, smin = 1.0, bound = 1.0;
      int nzero = 0;
#pragma unroll
      for (int c = 0; c < kGradNear; ++c) {
        const int k = nb[c];
        if (k < 0 || k == b) continue;
        const double R = Rb[k], d = __dsub_rn(db, nr[c]);
        if (d <= -__dmul_rn(kGradEdge, R)) continue;
        double q3, ds;
        becke_p3(__dmul_rn(d, Yb[k]), q3, ds);
        const double sv = __dmul_rn(0.5, __dsub_rn(1.0, q3));
        if (sv == 0.0) ++nzero;
        else Q *= sv;
        smin = fmin(smin, sv);
        bound = nzero == 0 ? (smin > 0.0 ? Q / smin : 0.0) : (nzero == 1 ? Q : 0.0);
        if (bound < kGradTau) break;
      }
      if (bound < kGradTau) {
        spnz[b * ld + p] = 0.0;
        snz[b * ld + p] = -2;
        continue;
      }
      double pnz = 1.0, fmin_row = 1.0;
      int nz = 0, zc = -1;
      for (int c = 0; c < natm; ++c) {
        if (c == b) continue;
        const double R = Rb[c], d = __dsub_rn(db, sd[c * ld + p]);
        if (d <= -__dmul_rn(kGradEdge, R)) continue;  // s == 1 exactly
        double q3, ds;
        becke_p3(__dmul_rn(d, Yb[c]), q3, ds);
        const double sv = __dmul_rn(0.5, __dsub_rn(1.0, q3));
        if (sv == 0.0) { ++nz; zc = c; }
        else { pnz *= sv; fmin_row = fmin(fmin_row, sv); }
      }
      // the largest leave-one-out product of the whole row decides: below tau the row is dead
      const double lmax = nz == 0 ? pnz / fmin_row : (nz == 1 ? pnz : 0.0);
      if (lmax < kGradTau) {
        spnz[b * ld + p] = 0.0;
        snz[b * ld + p] = -2;
        continue;
      }
      spnz[b * ld + p] = pnz;
      snz[b * ld + p] = nz == 0 ? -1 : zc;  // -1: no zero; c: the one zero; -2: dead
      if (b < 64) live_lo |= 1ull << b;
      else if (b < 128) live_hi |= 1ull << (b - 64);
      const double P = nz ? 0.0 : pnz;
      Z += P;
      if (b == h) Ph = P;
    }
    if (Z > 0.0) Wh = Ph / Z;
  }
  const bool go = live && Z > 0.0;
  const double iZ = go ? 1.0 / Z : 0.0;
  double gh[3] = {0, 0, 0};
  const int lane = threadIdx.x & 31;
  // rows live on some lane of the warp (MASK)
  uint64_t ulo = 0, uhi = 0;
  if (MASK) {
    const uint64_t mlo = go ? live_lo : 0ull, mhi = go ? live_hi : 0ull;
    ulo = ((uint64_t)__reduce_or_sync(0xffffffffu, (unsigned)(mlo >> 32)) << 32) |
          __reduce_or_sync(0xffffffffu, (unsigned)mlo);
    uhi = ((uint64_t)__reduce_or_sync(0xffffffffu, (unsigned)(mhi >> 32)) << 32) |
          __reduce_or_sync(0xffffffffu, (unsigned)mhi);
  }
  for (int x = 0; x < natm; ++x) {
    double gx[3] = {0, 0, 0};
    int zx = -2;
    double dx = 0.0, cx = 0.0, pnx = 0.0, ux[3] = {0, 0, 0};
    if (go) {
      dx = sd[x * ld + p];
      cx = e * ((x == h ? 1.0 : 0.0) - Wh) * iZ;
      const double ix = sinv[x * ld + p];
      for (int k = 0; k < 3; ++k) ux[k] = (rv[k] - atoms[3 * x + k]) * ix;
      if (!MASK || ((x < 64 ? live_lo >> x : live_hi >> (x - 64)) & 1ull)) {
        zx = snz[x * ld + p];
        pnx = spnz[x * ld + p];
      }
    }
    const bool lx = zx != -2;
    const double* Yx = rdist + (int64_t)x * natm;
    // a row x dead on every lane pairs only with rows live on some lane: walk
    // those (the same y in the same order as the full loop takes them)
    const bool xall = MASK && !__any_sync(0xffffffffu, lx);
    uint64_t ylo = xall ? ulo : ~0ull, yhi = xall ? uhi : ~0ull;
    for (int y = 0; y < natm; ++y) {
      if (MASK && xall) {
        if (ylo) {
          y = __ffsll((long long)ylo) - 1;
          ylo &= ylo - 1;
        } else if (yhi) {
          y = 64 + __ffsll((long long)yhi) - 1;
          yhi &= yhi - 1;
        } else {
          break;
        }
        if (y >= natm) break;
      }
      if (y == x) continue;
      int zy = -2;
      bool ly;
      if (MASK) {
        ly = ((y < 64 ? live_lo >> y : live_hi >> (y - 64)) & 1ull) != 0;
      } else {
        zy = go ? snz[y * ld + p] : -2;
        ly = zy != -2;
      }
      const bool need = go && (lx || ly);
      if (!__any_sync(0xffffffffu, need)) continue;
      if (!need) continue;
      if (MASK && ly) zy = snz[y * ld + p];
      const double iR = Yx[y];
      const double dy = sd[y * ld + p];
      const double mu = __dmul_rn(__dsub_rn(dx, dy), iR);
      double q3, ds;
      becke_p3(mu, q3, ds);
      const double sxy = __dmul_rn(0.5, __dsub_rn(1.0, q3)), syx = __dmul_rn(0.5, __dadd_rn(1.0, q3));
      // leave-one-out products of rows x (without y) and y (without x)
      const double Lxy = zx == -1 ? (sxy != 0.0 ? pnx / sxy : 0.0) : (zx == y ? pnx : 0.0);
      const double pny = spnz[y * ld + p];
      const double Lyx = zy == -1 ? (syx != 0.0 ? pny / syx : 0.0) : (zy == x ? pny : 0.0);
      const double cy = e * ((y == h ? 1.0 : 0.0) - Wh) * iZ;
      const double kxy = cx * Lxy * ds, kyx = cy * Lyx * ds;
      if (kxy == 0.0 && kyx == 0.0) continue;
      const double iy = sinv[y * ld + p];
      const double mr = mu * iR * iR;
      for (int k = 0; k < 3; ++k) {
        const double rxy = atoms[3 * x + k] - atoms[3 * y + k];
        const double uy = (rv[k] - atoms[3 * y + k]) * iy;
        gx[k] += (kyx - kxy) * (ux[k] * iR + mr * rxy);
        gh[k] += kxy * (ux[k] - uy) * iR;
      }
    }
    for (int k = 0; k < 3; ++k)
      for (int off = 16; off > 0; off >>= 1) gx[k] += __shfl_down_sync(0xffffffffu, gx[k], off);
    if (lane == 0)
      for (int k = 0; k < 3; ++k)
        if (gx[k] != 0.0) atomicAdd(&G[3 * x + k], gx[k]);
  }
  if (go)
    for (int k = 0; k < 3; ++k) atomicAdd(&G[3 * h + k], gh[k]);
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * natm; i += blockDim.x)
    if (G[i] != 0.0) atomicAdd(grad + i, G[i]);
}

// X (component 0) or Y_j (components 1..3) = (d_j Phi) P on the FP64 tensor
// pipe (DMMA): C[f][p] = sum_g A[g][p] P[g][f] for f < nbas, with the 64 x 64
// tile engine of dgemm.cuh (A: basis component rows of ld points, P: ldc x
// ldc, zero past nbas).  K runs to nbas rounded up to 16: the rows read past
// nbas belong to the next basis plane and meet P's zero rows.
__global__ void __launch_bounds__(kGemmThreads) k_grad_xy(const double* __restrict__ A, int64_t ld,
                                                         const double* __restrict__ P, int64_t ldc, int64_t nbas,
                                                         int64_t kend, double* __restrict__ C) {
  extern __shared__ double smem[];
  const int64_t m0 = (int64_t)blockIdx.x * 64, n0 = (int64_t)blockIdx.y * 64;
  Acc acc;
  acc.zero();
  gemm_tile<false, false>(acc, A, ld, m0, P, ldc, n0, 0, kend, smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t p = m0 + wm0 + i * 8 + (lane >> 2);
        const int64_t f = n0 + wn0 + j * 8 + 2 * (lane & 3) + e;
        if (f < nbas) C[f * ld + p] = acc.v[i][j][e];
      }
}

template <int L>
void launch_hess_l(const BuildArgs& a, int64_t p0, int64_t nvalid, int64_t ld, int64_t plane, double* out,
                   cudaStream_t st) {
  if (a.nshl[L] == 0) return;
  dim3 grid((unsigned)((ld + 127) / 128), (unsigned)a.nshl[L]);
  k_basis_hess<L><<<grid, 128, 0, st>>>(a.shells, a.shl[L], a.atoms, a.exps, a.norms, a.contr, a.rng, a.sa, a.px, a.py,
                                        a.pz, p0, nvalid, ld, plane, out);
}

}  // namespace

void launch_basis_hess(const BuildArgs& a, int64_t p0, int64_t nvalid, int64_t ld, int64_t plane, double* out,
                       cudaStream_t st) {
  launch_hess_l<0>(a, p0, nvalid, ld, plane, out, st);
  launch_hess_l<1>(a, p0, nvalid, ld, plane, out, st);
  launch_hess_l<2>(a, p0, nvalid, ld, plane, out, st);
  launch_hess_l<3>(a, p0, nvalid, ld, plane, out, st);
}

void launch_grad_points(const XcConst& K, int functional, bool gga, int ispin, int64_t nbas, int64_t ld, int64_t p0,
                        int64_t nvalid, const double* w, const double* wraw, const double* basis, int64_t plane,
                        const double* XY, double* coef, double* ef, double* exc, cudaStream_t st) {
  k_grad_points<<<(unsigned)((ld + 127) / 128), 128, 0, st>>>(K, functional, gga, ispin, nbas, ld, p0, nvalid, w,
                                                               wraw, basis, plane, XY, coef, ef, exc);
}

void launch_grad_orbital(bool gga, bool mgga, int ispin, int64_t nbas, int64_t ld, int64_t p0, int64_t nvalid,
                         int natm, const int* fatom, const int* owner, const double* basis, int64_t plane,
                         const double* XY, const double* coef, double* grad, cudaStream_t st) {
  const size_t smem = sizeof(double) * 3 * (kGradFB + natm);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_grad_orb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((unsigned)((nbas + kGradFB - 1) / kGradFB), (unsigned)((ld + 255) / 256));
  k_grad_orb<<<grid, 256, smem, st>>>(gga, mgga, ispin, nbas, ld, p0, nvalid, natm, fatom, owner, basis, plane, XY,
                                      coef, grad);
}

void launch_grad_w(int64_t nbas, int64_t ld, const double* basis, int64_t plane, const double* coef_b, double* W,
                   cudaStream_t st) {
  const int64_t n = round_up(nbas, 16) * ld;
  k_grad_w<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nbas, round_up(nbas, 16), ld, basis, plane, coef_b, W);
}

void launch_grad_xy(const double* basis_j, int64_t ld, const double* P, int64_t ldc, int64_t nbas, double* out,
                    cudaStream_t st) {
  constexpr int smem = gemm_smem_bytes<false, false>();
  cudaFuncSetAttribute(k_grad_xy, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const dim3 grid((unsigned)(ld / 64), (unsigned)((nbas + 63) / 64));
  k_grad_xy<<<grid, kGemmThreads, smem, st>>>(basis_j, ld, P, ldc, nbas, round_up(nbas, 16), out);
}

void launch_grad_weights(const double* atoms, const double* dist, int natm, const double* px, const double* py,
                         const double* pz, const int* owner, int64_t p0, int64_t nvalid, int64_t ld, const double* ef,
                         double* scratch, double* grad, cudaStream_t st) {
  if (nvalid <= 0) return;
  const size_t smem = sizeof(double) * 3 * natm;
  if (smem > 48 * 1024) {
    cudaFuncSetAttribute(k_grad_weights<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_grad_weights<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  const double* rdist = dist + (size_t)natm * natm;
  double* sd = scratch;
  double* sinv = scratch + (size_t)natm * ld;
  double* spnz = scratch + (size_t)2 * natm * ld;
  int* snz = (int*)(scratch + (size_t)3 * natm * ld);
  const unsigned nb = (unsigned)((nvalid + 127) / 128);
  if (natm <= 128)
    k_grad_weights<true><<<nb, 128, smem, st>>>(atoms, dist, rdist, natm, px, py, pz, owner, p0, nvalid, ld, ef, sd,
                                                sinv, spnz, snz, grad);
  else
    k_grad_weights<false><<<nb, 128, smem, st>>>(atoms, dist, rdist, natm, px, py, pz, owner, p0, nvalid, ld, ef, sd,
                                                 sinv, spnz, snz, grad);
}

}  // namespace pgxc
