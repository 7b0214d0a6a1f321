// xc_mgga.cuh -- meta-GGA functionals on the device: TPSS.
//
// TPSS as the reference's keyword evaluates it on the grid
// (modules/xc_func.f90:679-697): exchange of tpss_X (modules/tpss.f90,
// TPSS_key: tpss_exchange :243-428, mgga_inhomogeneity :431-617, get_*_var
// :619-815) and correlation of tpss_mgga_C (modules/tpss_mgga_module.f90
// :137-186, tpss :190-439: xc_z :443-487, co_c :684-801, pbe_c :805-896,
// co_e :900-1116), whose PBE pieces are pw_ldac (c_lda,
// modules/pw_ldac_module.f90:127-194) and gga_correlation with C_PBE
// (modules/gga_response_module.f90:170-420, H_pbe :585-600: beta =
// 0.06672455060314922).
//
// Derivatives by forward-mode duals: Dm<N> carries a value and N first
// derivatives; N = 3 for a closed shell (rho, gamma, tau), 7 for an open one
// (rho_a, rho_b, gamma_aa, gamma_bb, gamma_ab, tau_a, tau_b).  Where the
// reference sets a quantity to a constant outside a threshold, its
// derivatives are zero there.
#pragma once

#include <cuda_runtime.h>

namespace pgxc {
namespace mgga {

template <int N>
struct Dm {
  double v, d[N];
};
template <int N>
__device__ __forceinline__ Dm<N> mc(double x) {
  Dm<N> r;
  r.v = x;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dm<N> mv(int k, double x) {
  Dm<N> r = mc<N>(x);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = i == k ? 1.0 : 0.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dm<N> mf(const Dm<N>& a, double f, double df) {
  Dm<N> r;
  r.v = f;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dm<N> operator+(Dm<N> a, const Dm<N>& b) {
  a.v += b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) a.d[i] += b.d[i];
  return a;
}
template <int N>
__device__ __forceinline__ Dm<N> operator-(Dm<N> a, const Dm<N>& b) {
  a.v -= b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) a.d[i] -= b.d[i];
  return a;
}
template <int N>
__device__ __forceinline__ Dm<N> operator-(Dm<N> a) {
  a.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) a.d[i] = -a.d[i];
  return a;
}
template <int N>
__device__ __forceinline__ Dm<N> operator*(const Dm<N>& a, const Dm<N>& b) {
  Dm<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dm<N> operator/(const Dm<N>& a, const Dm<N>& b) {
  Dm<N> r;
  r.v = a.v / b.v;
  const double ib2 = 1.0 / (b.v * b.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * ib2;
  return r;
}
template <int N> __device__ __forceinline__ Dm<N> operator+(Dm<N> a, double b) { a.v += b; return a; }
template <int N> __device__ __forceinline__ Dm<N> operator+(double b, Dm<N> a) { a.v += b; return a; }
template <int N> __device__ __forceinline__ Dm<N> operator-(Dm<N> a, double b) { a.v -= b; return a; }
template <int N> __device__ __forceinline__ Dm<N> operator-(double b, const Dm<N>& a) { return mc<N>(b) - a; }
template <int N>
__device__ __forceinline__ Dm<N> operator*(Dm<N> a, double b) {
  a.v *= b;
#pragma unroll
  for (int i = 0; i < N; ++i) a.d[i] *= b;
  return a;
}
template <int N> __device__ __forceinline__ Dm<N> operator*(double b, const Dm<N>& a) { return a * b; }
template <int N> __device__ __forceinline__ Dm<N> operator/(const Dm<N>& a, double b) { return a * (1.0 / b); }
template <int N> __device__ __forceinline__ Dm<N> operator/(double b, const Dm<N>& a) { return mc<N>(b) / a; }
template <int N>
__device__ __forceinline__ Dm<N> mpow(const Dm<N>& a, double p) {
  const double v = pow(a.v, p);
  return mf(a, v, p * pow(a.v, p - 1.0));
}
template <int N> __device__ __forceinline__ Dm<N> msqrt(const Dm<N>& a) { const double s = sqrt(a.v); return mf(a, s, 0.5 / s); }
template <int N> __device__ __forceinline__ Dm<N> mexp(const Dm<N>& a) { const double e = exp(a.v); return mf(a, e, e); }
template <int N> __device__ __forceinline__ Dm<N> mlog(const Dm<N>& a) { return mf(a, log(a.v), 1.0 / a.v); }

constexpr double kPi = 3.14159265358979323846;

// PW92: n eps_c(na, nb) with the pw_ldac_module parameter sets
template <int N>
__device__ __forceinline__ Dm<N> pw92_G(const Dm<N>& rs, double a, double a1, double b1, double b2, double b3,
                                        double b4) {
  const Dm<N> sr = mpow(rs, 0.5);
  const Dm<N> q0 = -2.0 * a * (1.0 + a1 * rs);
  const Dm<N> q1 = 2.0 * a * (b1 * sr + b2 * rs + b3 * (rs * sr) + b4 * rs * rs);
  return q0 * mlog(1.0 + 1.0 / q1);
}
template <int N>
__device__ Dm<N> pw92_nec(const Dm<N>& na, const Dm<N>& nb) {
  const double deps = 1.0e-30;
  const double crs = pow(3.0 / (4.0 * 3.14159265358979324), 1.0 / 3.0);
  const double cf = 1.0 / (pow(2.0, 4.0 / 3.0) - 2.0);
  const double cfzz = 2.0 * (4.0 / 3.0) * (1.0 / 3.0) * cf;
  Dm<N> n = na + nb;
  if (n.v < deps) n = mc<N>(deps);
  const Dm<N> rs = crs / mpow(n, 1.0 / 3.0);
  const Dm<N> gu = pw92_G(rs, 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294);
  const Dm<N> gp = pw92_G(rs, 0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517);
  const Dm<N> ga = pw92_G(rs, 0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671);
  const Dm<N> z = (na - nb) / n;
  const Dm<N> z2 = z * z;
  const Dm<N> z4 = z2 * z2;
  const Dm<N> fz = cf * (mpow(1.0 + z + deps, 4.0 / 3.0) + mpow(1.0 - z + deps, 4.0 / 3.0) - 2.0);
  return n * (gu + (gp - gu) * fz * z4 - ga * fz * (1.0 - z4) / cfzz);
}

// n H of PBE correlation (gga_correlation, C_PBE); gm floored at 1e-20 for
// the spin-polarised branch; ec = pw92_nec of the same densities.
template <int N>
__device__ Dm<N> pbe_nh(const Dm<N>& na, const Dm<N>& nb, Dm<N> gm, const Dm<N>& ec, bool floor_gm) {
  const double eps = 1.0e-20;
  const double beta = 0.06672455060314922, gamma = 0.03109069086965489503494086371, bdg = beta / gamma;
  if (floor_gm && gm.v < eps) gm = mc<N>(eps);
  Dm<N> n = na + nb;
  if (fabs(n.v) < eps) n = mc<N>(eps);
  const Dm<N> z = (na - nb) / n;
  // spin scaling phi and its derivative with 1e-20 under the cube roots
  const double ph = 0.5 * (pow(1.0 + z.v, 2.0 / 3.0) + pow(1.0 - z.v, 2.0 / 3.0));
  const double dph = (1.0 / 3.0) * (pow(1.0 + z.v + eps, -1.0 / 3.0) - pow(1.0 - z.v + eps, -1.0 / 3.0));
  const Dm<N> phi = mf(z, ph, dph);
  const double t2f = kPi / (16.0 * pow(3.0 * kPi * kPi, 1.0 / 3.0));
  const Dm<N> den = phi * mpow(n, 7.0 / 6.0);
  const Dm<N> t2 = t2f * gm / (den * den);
  const Dm<N> phi3 = phi * phi * phi;
  const Dm<N> xe = -(ec / n) / (gamma * phi3);
  const Dm<N> A = xe.v <= 300.0 ? bdg / ((mexp(xe) - 1.0) + eps) : mc<N>(bdg / ((exp(xe.v) - 1.0) + eps));
  const Dm<N> at = A * t2;
  const Dm<N> g = bdg * t2 * ((1.0 + at) / (1.0 + at + at * at));
  return n * (gamma * phi3 * mlog(1.0 + g));
}

// eps_c^PBE per particle of pbe_c (zero below a density sum of 1e-9)
template <int N>
__device__ Dm<N> pbe_epc(const Dm<N>& na, const Dm<N>& nb, const Dm<N>& gm, const Dm<N>& sum, bool spin2) {
  if (sum.v < 1.0e-9) return mc<N>(0.0);
  const Dm<N> ec = pw92_nec(na, nb);
  return (pbe_nh(na, nb, gm, ec, spin2) + ec) / sum;
}

// TPSS exchange of one spin: e_x^LSDA(rho) F_x(x(rho, |grad rho|^2, tau))
template <int N>
__device__ Dm<N> tpss_xs(const Dm<N>& r, const Dm<N>& g, const Dm<N>& t) {
  const double tiny = 1.0e-40;
  const double kappa = 0.804, cpar = 1.59096, epar = 1.537, mupar = 0.21951, bpar = 0.40;
  if (!(r.v >= 1.0e-30)) return mc<N>(0.0);
  const Dm<N> ex = -0.930525736349100 * mpow(r, 4.0 / 3.0);
  const Dm<N> z = (r.v >= tiny && t.v >= tiny) ? g / (8.0 * r * t) : mc<N>(0.0);
  const Dm<N> p = r.v >= tiny ? g / (4.0 * pow(6.0 * kPi * kPi, 2.0 / 3.0) * mpow(r, 8.0 / 3.0)) : mc<N>(0.0);
  const Dm<N> al = r.v > tiny ? (t - g / (8.0 * r)) / (4.55779987234560 * mpow(r, 5.0 / 3.0)) : mc<N>(0.0);
  const Dm<N> qb = 0.45 * (al - 1.0) / msqrt(1.0 + bpar * al * (al - 1.0)) + (2.0 / 3.0) * p;
  const Dm<N> z2 = z * z;
  const Dm<N> d1 = 1.0 / (1.0 + z2);
  const Dm<N> zz = 0.6 * z;  // 3 z / 5
  const Dm<N> s2 = 0.5 * zz * zz + 0.5 * p * p;
  const Dm<N> s3 = sqrt(s2.v) > tiny ? msqrt(s2) : mc<N>(sqrt(s2.v));
  const double k81 = 10.0 / 81.0, se = sqrt(epar);
  Dm<N> num = (k81 + cpar * z2 * d1 * d1) * p;
  num = num + (146.0 / 2025.0) * qb * qb;
  num = num - (73.0 / 405.0) * s3 * qb;
  num = num + (k81 * k81 / kappa) * p * p;
  num = num + (2.0 * se * k81) * zz * zz;
  num = num + (epar * mupar) * p * p * p;
  const Dm<N> den = 1.0 + se * p;
  const Dm<N> x = num / (den * den);
  return ex * (1.0 + kappa - kappa / (1.0 + x / kappa));
}

// TPSS correlation energy per volume.  closed: the reference's ispin = 1
// path (C = 0.53), evaluated at equal spins.
template <int N>
__device__ Dm<N> tpss_cor(const Dm<N>& ra, const Dm<N>& rb, const Dm<N>& gaa, const Dm<N>& gbb, const Dm<N>& gab,
                          const Dm<N>& ta, const Dm<N>& tb, bool closed) {
  const double thld = 1.0e-9;
  const Dm<N> n = ra + rb;
  if (!(n.v >= thld)) return mc<N>(0.0);
  const Dm<N> gt = gaa + gbb + 2.0 * gab;
  const Dm<N> tt = ta + tb;
  const bool zon = tt.v >= thld;
  const Dm<N> zc = zon ? gt / (8.0 * n * tt) : mc<N>(1.0);
  const Dm<N> zc2 = zon ? zc * zc : mc<N>(1.0);
  const Dm<N> zero = mc<N>(0.0);
  const Dm<N> et = closed ? pbe_epc(0.5 * n, 0.5 * n, gt, n, false) : pbe_epc(ra, rb, gt, n, true);
  const Dm<N> ea = pbe_epc(ra, zero, gaa, ra, true);
  const Dm<N> pa = et.v >= ea.v ? et : ea;
  Dm<N> sumt, c;
  if (closed) {
    sumt = pa;
    c = mc<N>(0.53);
  } else {
    const Dm<N> eb = pbe_epc(rb, zero, gbb, rb, true);
    const Dm<N> pb = et.v >= eb.v ? et : eb;
    sumt = (ra * pa + rb * pb) / n;
    if (ra.v <= thld || rb.v <= thld) {
      c = mc<N>(0.0);
    } else {
      const Dm<N> rz = 1.0 / n;
      const Dm<N> zeta = (ra - rb) * rz;
      const Dm<N> zt2 = zeta * zeta;
      const Dm<N> xi2 = (rb * rb * gaa + ra * ra * gbb - 2.0 * ra * rb * gab) * (0.104484691940934 * mpow(rz, 14.0 / 3.0));
      const Dm<N> cn = 0.53 + (0.87 + (0.50 + 2.26 * zt2) * zt2) * zt2;
      const Dm<N> cd = 1.0 / (1.0 + 0.5 * xi2 * (mpow(1.0 + zeta, -4.0 / 3.0) + mpow(1.0 - zeta, -4.0 / 3.0)));
      const Dm<N> cd2 = cd * cd;
      c = cn * cd2 * cd2;
    }
  }
  const Dm<N> ep = et * (1.0 + c * zc2) - (1.0 + c) * zc2 * sumt;
  return n * (ep * (1.0 + 2.8 * ep * zc2 * zc));
}

// TPSS, closed shell: f and df/drho, df/dgamma, df/dtau of the total density
__device__ __forceinline__ void tpss_closed(double rho, double gam, double tau, double& f, double& fr, double& fg,
                                            double& ft) {
  const Dm<3> r = 0.5 * mv<3>(0, rho), g = 0.25 * mv<3>(1, gam), t = 0.5 * mv<3>(2, tau);
  const Dm<3> F = 2.0 * tpss_xs(r, g, t) + tpss_cor(r, r, g, g, g, t, t, true);
  f = F.v;
  fr = F.d[0];
  fg = F.d[1];
  ft = F.d[2];
}

// TPSS, open shell: rho (a, b), gam (aa, bb, ab), tau (a, b)
__device__ __forceinline__ void tpss_open(const double* rho, const double* gam, const double* tau, double& f,
                                          double* fr, double* fg, double* ft) {
  const Dm<7> ra = mv<7>(0, rho[0]), rb = mv<7>(1, rho[1]);
  const Dm<7> ga = mv<7>(2, gam[0]), gb = mv<7>(3, gam[1]), gc = mv<7>(4, gam[2]);
  const Dm<7> ta = mv<7>(5, tau[0]), tb = mv<7>(6, tau[1]);
  const Dm<7> F = tpss_xs(ra, ga, ta) + tpss_xs(rb, gb, tb) + tpss_cor(ra, rb, ga, gb, gc, ta, tb, false);
  f = F.v;
  fr[0] = F.d[0];
  fr[1] = F.d[1];
  fg[0] = F.d[2];
  fg[1] = F.d[3];
  fg[2] = F.d[4];
  ft[0] = F.d[5];
  ft[1] = F.d[6];
}

}  // namespace mgga
}  // namespace pgxc
