// xc_mgga.cuh -- meta-GGA functionals on the device: TPSS, VSXC, M06-L, M06.
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

#include "../../include/pgxc.h"

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

// ---------------------------------------------------------------------------
// VSXC (vsxc_mgga_module.f90) and the Minnesota M06-L / M06 (m06.f90):
// parameter set 0 VSXC, 1 M06-L, 2 M06 (grid part).  Per spin x^2 =
// gamma_ss / rho_s^(8/3) and z = 2 tau_s / rho_s^(5/3) - C_F (zero below
// 1e-30); h(x^2, z) the gvt4 form d0/g + (d1 x^2 + d2 z)/g^2 + (d3 x^4 + d4
// x^2 z + d5 z^2)/g^3, g = 1 + alpha (x^2 + z); D = 1 - x^2 / (4 (z + C_F))
// clipped at 0 (Dsic_term).
// ---------------------------------------------------------------------------
constexpr double kVsTol = 1.0e-30;
constexpr double kVsCF = 9.11559974469119;

struct VsPar {
  double dx[6];       // exchange h (gvt4, alpha 0.00186726)
  double dss[6];      // same-spin correlation h (alpha 0.00515088)
  double dos[6];      // opposite-spin correlation h (alpha 0.00304966)
  double a[12];       // M06 kinetic-energy series f(w) (sets 1, 2)
  double css[5], cos_[5];  // M06 B97-form series (beta 0.06 same spin, 0.0031 opposite)
};

__device__ __forceinline__ VsPar vs_par(int set) {
  VsPar P{};
  if (set == 0) {
    const double dx[6] = {1.05324147599106640E+00, 3.82234242542822070E-03, -6.71698348131996321E-03,
                          2.53030938105796706E-05, 1.37850244210630278E-04, -3.84172286736070984E-04};
    const double ds[6] = {3.270912E-01, -3.228915E-02, -2.942406E-02, 2.134222E-03, -5.451559E-03, 1.577575E-02};
    const double dd[6] = {7.035010E-01, 7.694574E-03, 5.152765E-02, 3.394308E-05, -1.269420E-03, 1.296118E-03};
    for (int i = 0; i < 6; ++i) { P.dx[i] = dx[i]; P.dss[i] = ds[i]; P.dos[i] = dd[i]; }
  } else if (set == 1) {
    const double dx[6] = {6.012244E-01, 4.748822E-03, -8.635108E-03, -9.308062E-06, 4.482811E-05, 0.0};
    const double ds[6] = {4.650534E-01, 1.617589E-01, 1.833657E-01, 4.692100E-04, -4.990573E-03, 0.0};
    const double dd[6] = {3.957626E-01, -5.614546E-01, 1.403963E-02, 9.831442E-04, -3.577176E-03, 0.0};
    const double a[12] = {3.987756E-01, 2.548219E-01, 3.923994E-01, -2.103655E+00, -6.302147E+00, 1.097615E+01,
                          3.097273E+01, -2.318489E+01, -5.673480E+01, 2.160364E+01, 3.421814E+01, -9.049762E+00};
    const double cs[5] = {5.349466E-01, 5.396620E-01, -3.161217E+01, 5.149592E+01, -2.919613E+01};
    const double co[5] = {6.042374E-01, 1.776783E+02, -2.513252E+02, 7.635173E+01, -1.255699E+01};
    for (int i = 0; i < 6; ++i) { P.dx[i] = dx[i]; P.dss[i] = ds[i]; P.dos[i] = dd[i]; }
    for (int i = 0; i < 12; ++i) P.a[i] = a[i];
    for (int i = 0; i < 5; ++i) { P.css[i] = cs[i]; P.cos_[i] = co[i]; }
  } else {
    const double dx[6] = {1.422057E-01, 7.370319E-04, -1.601373E-02, 0.0, 0.0, 0.0};
    const double ds[6] = {4.905945E-01, -1.437348E-01, 2.357824E-01, 1.871015E-03, -3.788963E-03, 0.0};
    const double dd[6] = {-2.741539E+00, -6.720113E-01, -7.932688E-02, 1.918681E-03, -2.032902E-03, 0.0};
    const double a[12] = {5.877943E-01, -1.371776E-01, 2.682367E-01, -2.515898E+00, -2.978892E+00, 8.710679E+00,
                          1.688195E+01, -4.489724E+00, -3.299983E+01, -1.449050E+01, 2.043747E+01, 1.256504E+01};
    const double cs[5] = {5.094055E-01, -1.491085E+00, 1.723922E+01, -3.859018E+01, 2.845044E+01};
    const double co[5] = {3.741539E+00, 2.187098E+02, -4.531252E+02, 2.936479E+02, -6.287470E+01};
    for (int i = 0; i < 6; ++i) { P.dx[i] = dx[i]; P.dss[i] = ds[i]; P.dos[i] = dd[i]; }
    for (int i = 0; i < 12; ++i) P.a[i] = a[i];
    for (int i = 0; i < 5; ++i) { P.css[i] = cs[i]; P.cos_[i] = co[i]; }
  }
  return P;
}

template <int N>
__device__ __forceinline__ Dm<N> vs_h(double alpha, const double* d, const Dm<N>& x2, const Dm<N>& z) {
  const Dm<N> g = 1.0 + alpha * (x2 + z);
  const Dm<N> ig = 1.0 / g;
  const Dm<N> ig2 = ig * ig;
  return d[0] * ig + (d[1] * x2 + d[2] * z) * ig2 + (d[3] * x2 * x2 + d[4] * x2 * z + d[5] * z * z) * (ig2 * ig);
}
template <int N>
__device__ __forceinline__ Dm<N> vs_x2(const Dm<N>& r, const Dm<N>& g) {
  return r.v >= kVsTol ? g / mpow(r, 8.0 / 3.0) : mc<N>(0.0);
}
template <int N>
__device__ __forceinline__ Dm<N> vs_zs(const Dm<N>& r, const Dm<N>& t) {
  return r.v >= kVsTol ? 2.0 * t / mpow(r, 5.0 / 3.0) - kVsCF : mc<N>(0.0);
}
template <int N>
__device__ __forceinline__ Dm<N> vs_D(const Dm<N>& r, const Dm<N>& g, const Dm<N>& t) {
  if (!(r.v >= kVsTol && t.v >= kVsTol)) return mc<N>(0.0);
  const Dm<N> D = 1.0 - (g / mpow(r, 8.0 / 3.0)) / (4.0 * (2.0 * t / mpow(r, 5.0 / 3.0)));
  return D.v < 0.0 ? mc<N>(0.0) : D;
}
template <int N>
__device__ __forceinline__ Dm<N> vs_ex(const Dm<N>& r) {
  return r.v >= kVsTol ? -0.930525736349100 * mpow(r, 4.0 / 3.0) : mc<N>(0.0);
}
template <int N>
__device__ __forceinline__ Dm<N> vs_series(double beta, const double* c, const Dm<N>& x2) {
  const Dm<N> v = beta * x2 / (1.0 + beta * x2);
  return c[0] + (c[1] + (c[2] + (c[3] + c[4] * v) * v) * v) * v;
}

// exchange of one spin: VSXC h, or M06 e_x F_PBE(x^2) f(w) plus the h term
template <int N>
__device__ Dm<N> vs_xs(int set, const VsPar& P, const Dm<N>& r, const Dm<N>& g, const Dm<N>& t) {
  const Dm<N> ex = vs_ex(r);
  const Dm<N> x2 = vs_x2(r, g);
  Dm<N> F = ex * vs_h(0.00186726, P.dx, x2, vs_zs(r, t));
  if (set > 0) {
    const Dm<N> fp = 1.0 + 3.612108584108E-03 * x2 / (1.0 + 4.49267E-3 * x2);
    Dm<N> w = mc<N>(0.0);
    if (r.v >= kVsTol && t.v >= kVsTol) {
      const Dm<N> tu = 4.55779987234560 * mpow(r, 5.0 / 3.0);
      w = (tu - t) / (tu + t);
    }
    Dm<N> k = mc<N>(P.a[11]);
    for (int j = 10; j >= 0; --j) k = k * w + P.a[j];
    F = F + ex * fp * k;
  }
  return F;
}

// correlation: the VSXC-form terms (a spin below 1e-30 has no derivatives
// there) and, for M06, the B97-form series
template <int N>
__device__ Dm<N> vs_cor(int set, const VsPar& P, const Dm<N>& ra0, const Dm<N>& rb0, const Dm<N>& gaa,
                        const Dm<N>& gbb, const Dm<N>& ta, const Dm<N>& tb) {
  const Dm<N> zero = mc<N>(0.0);
  Dm<N> F = zero;
  {
    const Dm<N> ra = ra0.v >= kVsTol ? ra0 : mc<N>(ra0.v);
    const Dm<N> rb = rb0.v >= kVsTol ? rb0 : mc<N>(rb0.v);
    const Dm<N> ea = pw92_nec(ra, zero), eb = pw92_nec(zero, rb);
    const Dm<N> eo = pw92_nec(ra, rb) - ea - eb;
    if (ra.v >= kVsTol) F = F + ea * vs_h(0.00515088, P.dss, vs_x2(ra, gaa), vs_zs(ra, ta)) * vs_D(ra, gaa, ta);
    if (rb.v >= kVsTol) F = F + eb * vs_h(0.00515088, P.dss, vs_x2(rb, gbb), vs_zs(rb, tb)) * vs_D(rb, gbb, tb);
    if ((ra + rb).v >= kVsTol)
      F = F + eo * vs_h(0.00304966, P.dos, vs_x2(ra, gaa) + vs_x2(rb, gbb), vs_zs(ra, ta) + vs_zs(rb, tb));
  }
  if (set > 0) {
    const Dm<N> ea = pw92_nec(ra0, zero), eb = pw92_nec(zero, rb0);
    const Dm<N> eo = pw92_nec(ra0, rb0) - ea - eb;
    const Dm<N> xa = vs_x2(ra0, gaa), xb = vs_x2(rb0, gbb);
    F = F + ea * vs_series(0.06, P.css, xa) * vs_D(ra0, gaa, ta);
    F = F + eb * vs_series(0.06, P.css, xb) * vs_D(rb0, gbb, tb);
    F = F + eo * vs_series(0.0031, P.cos_, xa + xb);
  }
  return F;
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

// Any meta-GGA keyword, closed shell.  The open-shell form at rho/2, gamma/4,
// tau/2; VSXC's closed-shell derivatives are half the chain rule, as the
// reference's vsxc_X / vsxc_C wrappers return them.
__device__ __forceinline__ void mgga_closed(int functional, double rho, double gam, double tau, double& f,
                                            double& fr, double& fg, double& ft) {
  if (functional == PGXC_XC_TPSS) {
    tpss_closed(rho, gam, tau, f, fr, fg, ft);
    return;
  }
  const int set = functional == PGXC_XC_VSXC ? 0 : functional == PGXC_XC_M06L ? 1 : 2;
  const VsPar P = vs_par(set);
  const Dm<3> r = 0.5 * mv<3>(0, rho), g = 0.25 * mv<3>(1, gam), t = 0.5 * mv<3>(2, tau);
  const Dm<3> F = 2.0 * vs_xs(set, P, r, g, t) + vs_cor(set, P, r, r, g, g, t, t);
  const double h = set == 0 ? 0.5 : 1.0;
  f = F.v;
  fr = h * F.d[0];
  fg = h * F.d[1];
  ft = h * F.d[2];
}

// Any meta-GGA keyword, open shell
__device__ __forceinline__ void mgga_open(int functional, const double* rho, const double* gam, const double* tau,
                                          double& f, double* fr, double* fg, double* ft) {
  if (functional == PGXC_XC_TPSS) {
    tpss_open(rho, gam, tau, f, fr, fg, ft);
    return;
  }
  const int set = functional == PGXC_XC_VSXC ? 0 : functional == PGXC_XC_M06L ? 1 : 2;
  const VsPar P = vs_par(set);
  const Dm<6> ra = mv<6>(0, rho[0]), rb = mv<6>(1, rho[1]);
  const Dm<6> ga = mv<6>(2, gam[0]), gb = mv<6>(3, gam[1]);
  const Dm<6> ta = mv<6>(4, tau[0]), tb = mv<6>(5, tau[1]);
  const Dm<6> F = vs_xs(set, P, ra, ga, ta) + vs_xs(set, P, rb, gb, tb) + vs_cor(set, P, ra, rb, ga, gb, ta, tb);
  f = F.v;
  fr[0] = F.d[0];
  fr[1] = F.d[1];
  fg[0] = F.d[2];
  fg[1] = F.d[3];
  fg[2] = 0.0;  // gamma_ab does not enter VSXC or M06
  ft[0] = F.d[4];
  ft[1] = F.d[5];
}

}  // namespace mgga
}  // namespace pgxc
