// basis.cuh -- contracted real-solid-harmonic Gaussians and gradients on points.
//
// Restates, per point and per (atom, l) shell:
//   solid_harmonics_calculate  modules/solid_harmonics_module.f90:369-482
//     (Racah-normalised recursion, Y_00 = 1, Y_1 = (z, x, y)); the gradients
//     of :488-568 are obtained by differentiating the same recursion;
//   radial                     modules/orbital_module.f90:1742-1932
//     (norm*exp(-a r^2) only where a r^2 < 50, derivative factor -2a, the
//     first N_uncontracted primitives bare, then the contractions);
//   calculate_orbs_and_grads_v3 modules/orbital_module.f90:2421-2619
//     (phi = Y R, grad phi = (r - R_A) Y R' + grad(Y) R; function order
//     independent function -> radial function).
#pragma once

#include "pgxc_common.cuh"

namespace pgxc {

// Y[l*l + m] and dY[c][l*l + m], c = x, y, z, for l <= L.
template <int L>
__device__ __forceinline__ void solid_harmonics(double x, double y, double z, double* Y, double (*dY)[16]) {
  const double r2 = x * x + y * y + z * z;
  Y[0] = 1.0;
  dY[0][0] = dY[1][0] = dY[2][0] = 0.0;
  if (L == 0) return;
  Y[1] = z; Y[2] = x; Y[3] = y;
  dY[0][1] = 0; dY[1][1] = 0; dY[2][1] = 1;
  dY[0][2] = 1; dY[1][2] = 0; dY[2][2] = 0;
  dY[0][3] = 0; dY[1][3] = 1; dY[2][3] = 0;
#pragma unroll
  for (int l = 2; l <= L; ++l) {
    const int o = l * l, o1 = (l - 1) * (l - 1), o2 = (l - 2) * (l - 2);
    const double lr = l, l1r = l - 1, ll1r = 2 * l - 1;
    const double dr2[3] = {2 * x, 2 * y, 2 * z};
    // m index 0
    {
      const double p1 = Y[o1], p2 = Y[o2];
      Y[o] = (ll1r * z * p1 - l1r * r2 * p2) / lr;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        dY[c][o] = (ll1r * ((c == 2 ? p1 : 0.0) + z * dY[c][o1]) - l1r * (dr2[c] * p2 + r2 * dY[c][o2])) / lr;
    }
#pragma unroll
    for (int im = 1; im <= l - 2; ++im) {
      const double sim = (double)(im * im);
      const double rlm = 1.0 / sqrt(lr * lr - sim);
      const double rl1m = sqrt(l1r * l1r - sim);
      const double a = ll1r * z * rlm;
      const double b = rl1m * r2 * rlm;
#pragma unroll
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const double p1 = Y[o1 + mm], p2 = Y[o2 + mm];
        Y[o + mm] = a * p1 - b * p2;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : 0.0) + a * dY[c][o1 + mm] - rl1m * dr2[c] * rlm * p2 -
                          b * dY[c][o2 + mm];
      }
    }
    {
      const int im = l - 1;
      const double rlm = 1.0 / sqrt(lr * lr - (double)(im * im));
      const double a = ll1r * z * rlm;
#pragma unroll
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const double p1 = Y[o1 + mm];
        Y[o + mm] = a * p1;
#pragma unroll
        for (int c = 0; c < 3; ++c) dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : 0.0) + a * dY[c][o1 + mm];
      }
    }
    {
      const double rll = sqrt(ll1r / (2 * lr));
      const double q2 = Y[o1 + 2 * l - 3], q1 = Y[o1 + 2 * l - 2];
      Y[o + 2 * l - 1] = (x * q2 - y * q1) * rll;
      Y[o + 2 * l] = (y * q2 + x * q1) * rll;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double g2 = dY[c][o1 + 2 * l - 3], g1 = dY[c][o1 + 2 * l - 2];
        const double dx = (c == 0), dy = (c == 1);
        dY[c][o + 2 * l - 1] = (dx * q2 + x * g2 - dy * q1 - y * g1) * rll;
        dY[c][o + 2 * l] = (dy * q2 + y * g2 + dx * q1 + x * g1) * rll;
      }
    }
  }
}

// Output element types: FP64 for the drop-in path, FP32 for the mixed path.
template <typename T>
__device__ __forceinline__ T cvt_out(double v) { return (T)v; }

// Evaluate one shell at one point and store its (2l+1)*nrad functions (and
// gradients when GRAD) at column p of the [function][ld] arrays.
template <int L, bool GRAD, typename T>
__device__ __forceinline__ void shell_at_point(const DevShell& S, const DevSA& sa, double x, double y, double z,
                                               const double* __restrict__ exps, const double* __restrict__ norms,
                                               const double* __restrict__ contr, bool valid, int64_t p, int64_t ld,
                                               T* __restrict__ phi, T* __restrict__ gx, T* __restrict__ gy,
                                               T* __restrict__ gz) {
  constexpr int NY = (L + 1) * (L + 1);
  double Y[16];
  double dY[3][16];
  solid_harmonics<L>(x, y, z, Y, dY);
  const double r2 = x * x + y * y + z * z;
  // symmetry-adapted harmonics of this l
  double Ys[2 * L + 1], dYs[3][2 * L + 1];
#pragma unroll
  for (int i = 0; i < 2 * L + 1; ++i) {
    if (sa.identity) {
      Ys[i] = Y[L * L + i];
#pragma unroll
      for (int c = 0; c < 3; ++c) dYs[c][i] = dY[c][L * L + i];
    } else {
      double v = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m) {
        const double cf = sa.c[L][i][m];
        v += cf * Y[L * L + m];
        g0 += cf * dY[0][L * L + m];
        g1 += cf * dY[1][L * L + m];
        g2 += cf * dY[2][L * L + m];
      }
      Ys[i] = v; dYs[0][i] = g0; dYs[1][i] = g1; dYs[2][i] = g2;
    }
  }
  (void)NY;
  const double* ex = exps + S.exp_off;
  const double* nr = norms + S.exp_off;
  const double* cc = contr + S.con_off;
  for (int r0 = 0; r0 < S.nrad; r0 += kRadGroup) {
    double R[kRadGroup], dR[kRadGroup];
#pragma unroll
    for (int r = 0; r < kRadGroup; ++r) { R[r] = 0.0; dR[r] = 0.0; }
    if (valid) {
      for (int e = 0; e < S.nexp; ++e) {
        const double alpha = __ldg(ex + e);
        const double ar2 = alpha * r2;
        double v = 0.0;
        if (ar2 < 50.0) v = __ldg(nr + e) * exp(-ar2);
        const double dv = (-2.0 * alpha) * v;
#pragma unroll
        for (int r = 0; r < kRadGroup; ++r) {
          const int rr = r0 + r;
          if (rr < S.nrad) {
            double cf;
            if (rr < S.nunc) cf = (e == rr) ? 1.0 : 0.0;
            else cf = __ldg(cc + e + (int64_t)S.nexp * (rr - S.nunc));
            R[r] += cf * v;
            dR[r] += cf * dv;
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 2 * L + 1; ++i) {
#pragma unroll
      for (int r = 0; r < kRadGroup; ++r) {
        const int rr = r0 + r;
        if (rr < S.nrad) {
          const int64_t f = S.f0 + (int64_t)i * S.nrad + rr;
          phi[f * ld + p] = cvt_out<T>(Ys[i] * R[r]);
          if (GRAD) {
            const double h = Ys[i] * dR[r];
            gx[f * ld + p] = cvt_out<T>(x * h + dYs[0][i] * R[r]);
            gy[f * ld + p] = cvt_out<T>(y * h + dYs[1][i] * R[r]);
            gz[f * ld + p] = cvt_out<T>(z * h + dYs[2][i] * R[r]);
          }
        }
      }
    }
  }
}

}  // namespace pgxc
