// mgga_oracle.h -- the meta-GGA functionals of the CPU oracle (test
// infrastructure only: nothing in the library links or calls it).
//
// TPSS, as the reference's keyword "TPSS" evaluates it on the grid
// (xc_func.f90:679-697): exchange by tpss_X of modules/tpss.f90 (TPSS_key,
// :110-189 with tpss_exchange :243-428, mgga_inhomogeneity :431-617 and the
// get_*_var helpers :619-815) and correlation by tpss_mgga_C of
// modules/tpss_mgga_module.f90 (:137-186 through tpss :190-439 with corron:
// xc_z :443-487, co_c :684-801, pbe_c :805-896, co_e :900-1116).  pbe_c takes
// the LDA part from pw_ldac (modules/pw_ldac_module.f90:197-312, c_lda) and
// the gradient part from gga_correlation with C_PBE
// (modules/gga_response_module.f90:170-275, pbe_or_pw91 :278-420, H_pbe
// :585-600, H0_drv, A_drv, Hln_drv).
//
// The energies are restated in forward-mode dual numbers (DN<N>: a value and
// N first derivatives); the reference's hand-written derivative formulas are
// the derivatives of the same expressions.  Branches follow the reference's
// WHERE masks: a quantity set to a constant in a masked-out branch has zero
// derivatives there.
#pragma once

#include <cmath>

namespace mgga {

template <int N>
struct DN {
  double v;
  double d[N];
};
template <int N>
inline DN<N> cst(double x) {
  DN<N> r;
  r.v = x;
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
inline DN<N> var(int i, double x) {
  DN<N> r = cst<N>(x);
  r.d[i] = 1.0;
  return r;
}
// f(a) with f(a.v) = fv and f'(a.v) = df
template <int N>
inline DN<N> chain(const DN<N>& a, double fv, double df) {
  DN<N> r;
  r.v = fv;
  for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
  return r;
}
template <int N>
inline DN<N> operator+(DN<N> a, const DN<N>& b) {
  a.v += b.v;
  for (int i = 0; i < N; ++i) a.d[i] += b.d[i];
  return a;
}
template <int N>
inline DN<N> operator-(DN<N> a, const DN<N>& b) {
  a.v -= b.v;
  for (int i = 0; i < N; ++i) a.d[i] -= b.d[i];
  return a;
}
template <int N>
inline DN<N> operator-(DN<N> a) {
  a.v = -a.v;
  for (int i = 0; i < N; ++i) a.d[i] = -a.d[i];
  return a;
}
template <int N>
inline DN<N> operator*(const DN<N>& a, const DN<N>& b) {
  DN<N> r;
  r.v = a.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
inline DN<N> operator/(const DN<N>& a, const DN<N>& b) {
  DN<N> r;
  r.v = a.v / b.v;
  const double q = b.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / q;
  return r;
}
template <int N> inline DN<N> operator+(DN<N> a, double b) { a.v += b; return a; }
template <int N> inline DN<N> operator+(double b, DN<N> a) { a.v += b; return a; }
template <int N> inline DN<N> operator-(DN<N> a, double b) { a.v -= b; return a; }
template <int N> inline DN<N> operator-(double b, const DN<N>& a) { return cst<N>(b) - a; }
template <int N>
inline DN<N> operator*(DN<N> a, double b) {
  a.v *= b;
  for (int i = 0; i < N; ++i) a.d[i] *= b;
  return a;
}
template <int N> inline DN<N> operator*(double b, const DN<N>& a) { return a * b; }
template <int N> inline DN<N> operator/(const DN<N>& a, double b) { return a * (1.0 / b) ; }
template <int N> inline DN<N> operator/(double b, const DN<N>& a) { return cst<N>(b) / a; }
template <int N>
inline DN<N> dpow(const DN<N>& a, double p) {
  return chain(a, std::pow(a.v, p), p * std::pow(a.v, p - 1.0));
}
template <int N> inline DN<N> dsqrt(const DN<N>& a) { const double s = std::sqrt(a.v); return chain(a, s, 0.5 / s); }
template <int N> inline DN<N> dexp(const DN<N>& a) { const double e = std::exp(a.v); return chain(a, e, e); }
template <int N> inline DN<N> dlog(const DN<N>& a) { return chain(a, std::log(a.v), 1.0 / a.v); }

const double PI = 3.14159265358979323846;

// PW92 c_lda(na, nb) = n eps_c (pw_ldac_module.f90:127-194, set_param
// :591-651, non-RPA): the same arithmetic as the oracle's 3-variable copy.
template <int N>
DN<N> pw92_g(const DN<N>& rs, int what) {
  double a, a1, b1, b2, b3, b4;
  if (what == 1) { a = 0.031091; a1 = 0.21370; b1 = 7.5957; b2 = 3.5876; b3 = 1.6382; b4 = 0.49294; }
  else if (what == 2) { a = 0.015545; a1 = 0.20548; b1 = 14.1189; b2 = 6.1977; b3 = 3.3662; b4 = 0.62517; }
  else { a = 0.016887; a1 = 0.11125; b1 = 10.357; b2 = 3.6231; b3 = 0.88026; b4 = 0.49671; }
  const DN<N> rs1d2 = dpow(rs, 0.5);
  const DN<N> Q0 = -2.0 * a * (1.0 + a1 * rs);
  const DN<N> Q1 = 2.0 * a * (b1 * rs1d2 + b2 * rs + b3 * (rs * rs1d2) + b4 * rs * dpow(rs, 1.0));
  return Q0 * dlog(1.0 + 1.0 / Q1);
}
template <int N>
DN<N> pw92_c_lda(const DN<N>& na, const DN<N>& nb) {
  const double deps = 1.0e-30, pi = 3.14159265358979324;
  const double c1d3 = 1.0 / 3.0, c4d3 = 4.0 / 3.0;
  const double crs = std::pow(3.0 / (4.0 * pi), c1d3);
  const double cf = 1.0 / (std::pow(2.0, c4d3) - 2.0);
  const double cfzz = 2.0 * c4d3 * c1d3 * cf;
  DN<N> nn = na + nb;
  if (nn.v < deps) nn = cst<N>(deps);
  const DN<N> rs = crs / dpow(nn, c1d3);
  const DN<N> ecu = pw92_g(rs, 1), ecp = pw92_g(rs, 2), malf = pw92_g(rs, 3);
  const DN<N> z = (na - nb) / nn;
  const DN<N> z2 = z * z;
  const DN<N> z4 = z2 * z2;
  const DN<N> f = cf * (dpow(1.0 + z + deps, c4d3) + dpow(1.0 - z + deps, c4d3) - 2.0);
  return nn * (ecu + (ecp - ecu) * f * z4 - malf * f * (1.0 - z4) / cfzz);
}

// n H of the PBE correlation, gga_correlation / pbe_or_pw91 with C_PBE:
// na, nb the spin densities, gm |grad n|^2 (floored at 1e-20 for ispin 2),
// ec the LDA correlation energy per volume of pw_ldac.
template <int N>
DN<N> pbe_nH(DN<N> na, DN<N> nb, DN<N> gm, const DN<N>& ec, bool floor_gm) {
  const double eps = 1.0e-20, pi = 3.14159265358979324;
  const double beta = 0.06672455060314922, gamma = 0.03109069086965489503494086371, bdg = beta / gamma;
  if (floor_gm && gm.v < eps) gm = cst<N>(eps);
  DN<N> nn = na + nb;
  if (std::fabs(nn.v) < eps) nn = cst<N>(eps);
  const DN<N> z = (na - nb) / nn;
  // phi = ((1+z)^(2/3) + (1-z)^(2/3)) / 2; its derivative with 1e-20 under
  // the cube roots (pbe_or_pw91, dphidz)
  const double c2d3 = 2.0 / 3.0, c1d3 = 1.0 / 3.0;
  const double phv = 0.5 * (std::pow(1.0 + z.v, c2d3) + std::pow(1.0 - z.v, c2d3));
  const double dph = c1d3 * (std::pow(1.0 + z.v + eps, -c1d3) - std::pow(1.0 - z.v + eps, -c1d3));
  const DN<N> phi = chain(z, phv, dph);
  const double t2_fact = pi / (4.0 * 4.0 * std::pow(3.0 * pi * pi, c1d3));
  const DN<N> den = phi * dpow(nn, 7.0 / 6.0);
  const DN<N> t = t2_fact * gm / (den * den);  // t^2
  const DN<N> Flda = ec / nn;
  // A_drv: A = bdg / (exp(-e / (gamma phi^3)) - 1 + eps), derivatives zero where the exponent is above 300
  const DN<N> p3 = phi * phi * phi;
  const DN<N> Xe = -Flda / (gamma * p3);
  DN<N> A;
  if (Xe.v <= 300.0) A = bdg / ((dexp(Xe) - 1.0) + eps);
  else A = cst<N>(bdg / ((std::exp(Xe.v) - 1.0) + eps));
  // Hln_drv: H = log(1 + g), g = bdg t (1 + A t) / (1 + A t + (A t)^2)
  const DN<N> At = 1.0 + A * t;
  const DN<N> At2 = At + (A * t) * (A * t);
  const DN<N> g = bdg * t * (At / At2);
  return nn * (gamma * p3 * dlog(1.0 + g));
}

// eps_c^PBE per particle as pbe_c: (n H + c_lda) / sum rho for sum rho >=
// 1e-9, else 0.  spin: the gga_correlation branch (1: n/2, n/2 with |grad
// n|^2 as given; 2: spin densities with the 1e-20 floor).
template <int N>
DN<N> pbe_eps(const DN<N>& na, const DN<N>& nb, const DN<N>& gm, const DN<N>& sumrho, int spin) {
  const double thld = 1.0e-9;
  if (sumrho.v < thld) return cst<N>(0.0);
  const DN<N> ec = pw92_c_lda(na, nb);
  return (pbe_nH(na, nb, gm, ec, spin == 2) + ec) / sumrho;
}

// TPSS exchange of one spin density (tpss_exchange with exchef and
// mgga_inhomogeneity, TPSS_key): e_x^LSDA(rho_s) F_x(x), rho, |grad rho|^2
// and tau of that spin.
template <int N>
DN<N> tpss_x_spin(const DN<N>& rho, const DN<N>& gr2, const DN<N>& tau) {
  const double DTol = 1.0e-40, DTolX = 1.0e-30;
  const double kappa = 0.804, c_par = 1.59096, e_par = 1.537, mupar = 0.21951, b_par = 0.40;
  const double CX = -0.930525736349100, CT = 4.55779987234560;
  if (!(rho.v >= DTolX)) return cst<N>(0.0);  // eX_lsda: e = 0 below 1e-30
  const DN<N> e = CX * dpow(rho, 4.0 / 3.0);
  const DN<N> z = (rho.v >= DTol && tau.v >= DTol) ? gr2 / (8.0 * rho * tau) : cst<N>(0.0);
  const DN<N> p = rho.v >= DTol
                      ? gr2 / (4.0 * std::pow(6.0 * PI * PI, 2.0 / 3.0) * dpow(rho, 8.0 / 3.0))
                      : cst<N>(0.0);
  const DN<N> a = rho.v > DTol ? (tau - gr2 / (8.0 * rho)) / (CT * dpow(rho, 5.0 / 3.0)) : cst<N>(0.0);
  const DN<N> q = 0.45 * (a - 1.0) * (1.0 / dsqrt(1.0 + b_par * a * (a - 1.0))) + (2.0 / 3.0) * p;
  const DN<N> d1 = 1.0 / (1.0 + z * z);
  const DN<N> t1 = (10.0 / 81.0 + c_par * z * z * d1 * d1) * p;
  const DN<N> t2 = (146.0 / 2025.0) * q * q;
  const DN<N> z35 = 3.0 * z / 5.0;
  const DN<N> s3sq = 0.5 * z35 * z35 + 0.5 * p * p;
  const double s3v = std::sqrt(s3sq.v);
  // t3 = -(73/405) s3 q; the reference's derivatives of s3 are zero where s3 <= 1e-40
  const DN<N> s3 = s3v > DTol ? dsqrt(s3sq) : cst<N>(s3v);
  const DN<N> t3 = -(73.0 / 405.0) * s3 * q;
  const DN<N> t4 = (1.0 / kappa) * (10.0 / 81.0) * (10.0 / 81.0) * p * p;
  const DN<N> t5 = 2.0 * std::sqrt(e_par) * (10.0 / 81.0) * z35 * z35;
  const DN<N> t6 = e_par * mupar * p * p * p;
  const DN<N> t7 = 1.0 + std::sqrt(e_par) * p;
  const DN<N> x = (t1 + t2 + t3 + t4 + t5 + t6) / (t7 * t7);
  const DN<N> f = 1.0 + kappa - kappa / (1.0 + x / kappa);
  return e * f;
}

// TPSS correlation energy per volume (tpss with corron, co_e, co_c, xc_z) of
// the spin densities, their gradient products and kinetic energy densities.
// closed: the reference's ispin = 1 path (C(zeta, xi) = 0.53), evaluated at
// na = nb, gaa = gbb = gab, ta = tb.
template <int N>
DN<N> tpss_c(const DN<N>& ra, const DN<N>& rb, const DN<N>& gaa, const DN<N>& gbb, const DN<N>& gab,
             const DN<N>& ta, const DN<N>& tb, bool closed) {
  const double thld = 1.0e-9, d_H = 2.8;
  const double c0 = 0.53, c2 = 0.87, c4 = 0.50, c6 = 2.26, cx = 0.104484691940934;
  const DN<N> sumrho = ra + rb;
  const DN<N> sumgam = gaa + gbb + 2.0 * gab;
  const DN<N> sumtau = ta + tb;
  if (!(sumrho.v >= thld)) return cst<N>(0.0);  // epsPKZB = 0
  // xc_z of the total density: 1 (constant) where rho or tau is below 1e-9
  const bool zon = sumrho.v >= thld && sumtau.v >= thld;
  const DN<N> zc = zon ? sumgam / (8.0 * sumrho * sumtau) : cst<N>(1.0);
  const DN<N> zc2 = zon ? zc * zc : cst<N>(1.0);
  // PBE of the total density and of each spin alone (co_e)
  const DN<N> zero = cst<N>(0.0);
  const DN<N> f_t = closed ? pbe_eps(0.5 * sumrho, 0.5 * sumrho, sumgam, sumrho, 1)
                           : pbe_eps(ra, rb, sumgam, sumrho, 2);
  DN<N> epst[2];
  const DN<N>* rs[2] = {&ra, &rb};
  const DN<N>* gs[2] = {&gaa, &gbb};
  for (int s = 0; s < (closed ? 1 : 2); ++s) {
    const DN<N> f_s = pbe_eps(*rs[s], zero, *gs[s], *rs[s], 2);
    epst[s] = f_t.v >= f_s.v ? f_t : f_s;
  }
  DN<N> sumt;
  if (closed) sumt = epst[0];
  else sumt = (ra * epst[0] + rb * epst[1]) / sumrho;
  // C(zeta, xi), co_c
  DN<N> c;
  if (closed) {
    c = cst<N>(c0);
  } else if (ra.v <= thld || rb.v <= thld || sumrho.v <= thld) {
    c = cst<N>(0.0);
  } else {
    const DN<N> rez = 1.0 / sumrho;
    const DN<N> av4 = cx * dpow(rez, 14.0 / 3.0);
    const DN<N> zeta = (ra - rb) * rez;
    const DN<N> zet2 = zeta * zeta;
    const DN<N> xi2 = (rb * rb * gaa + ra * ra * gbb - 2.0 * ra * rb * gab) * av4;
    const DN<N> cn = c0 + (c2 + (c4 + c6 * zet2) * zet2) * zet2;
    const DN<N> cd = 1.0 / (1.0 + 0.5 * xi2 * (dpow(1.0 + zeta, -4.0 / 3.0) + dpow(1.0 - zeta, -4.0 / 3.0)));
    const DN<N> cd2 = cd * cd;
    c = cn * cd2 * cd2;
  }
  const DN<N> epk = f_t * (1.0 + c * zc2) - (1.0 + c) * zc2 * sumt;
  const DN<N> etp = epk * (1.0 + d_H * epk * zc2 * zc);
  return sumrho * etp;
}

// ---------------------------------------------------------------------------
// VSXC and the Minnesota M06 family: modules/vsxc_mgga_module.f90 (vsxc_X
// :90-173, vsxc_C :177-260, vsxc_exchange :264-425, vsxc_correlation
// :429-722, eX_lsda :726-762, Dsic_term :766-850, gvt4_term :854-975) and
// modules/m06.f90 (m06_X :85-156, m06_C :160-231, m06_exchange :235-563 with
// pbeef and kedef, m06_correlation :567-821, bmk_term :825-906).  Parameter
// set 0 is VSXC, 1 M06-L, 2 M06 (the grid part of the hybrid).
// ---------------------------------------------------------------------------
const double VS_DTOL = 1.0e-30;
const double VS_CF = 9.11559974469119;

// gvt4_term's h(x^2, z) = d0/g + (d1 x^2 + d2 z)/g^2 + (d3 x^4 + d4 x^2 z + d5 z^2)/g^3, g = 1 + alpha (x^2 + z)
template <int N>
DN<N> gvt4(double alpha, const double* d, const DN<N>& x2, const DN<N>& z) {
  const DN<N> g = 1.0 + alpha * (x2 + z);
  const DN<N> g2 = g * g;
  return d[0] / g + (d[1] * x2 + d[2] * z) / g2 + (d[3] * x2 * x2 + d[4] * x2 * z + d[5] * z * z) / (g2 * g);
}
// x_s^2 = gamma_ss / rho_s^(8/3) and z_s = 2 tau_s / rho_s^(5/3) - CF; zero below 1e-30
template <int N>
DN<N> vs_x2(const DN<N>& r, const DN<N>& g) {
  return r.v >= VS_DTOL ? g / dpow(r, 8.0 / 3.0) : cst<N>(0.0);
}
template <int N>
DN<N> vs_z(const DN<N>& r, const DN<N>& t) {
  return r.v >= VS_DTOL ? 2.0 * t / dpow(r, 5.0 / 3.0) - VS_CF : cst<N>(0.0);
}
// Dsic_term: 1 - x^2 / (4 (z + CF)) where rho and tau are above 1e-30, clipped at 0
template <int N>
DN<N> vs_dsic(const DN<N>& r, const DN<N>& g, const DN<N>& t) {
  if (!(r.v >= VS_DTOL && t.v >= VS_DTOL)) return cst<N>(0.0);
  const DN<N> x2 = g / dpow(r, 8.0 / 3.0);
  const DN<N> z = 2.0 * t / dpow(r, 5.0 / 3.0) - VS_CF;
  const DN<N> D = 1.0 - x2 / (4.0 * (z + VS_CF));
  return D.v < 0.0 ? cst<N>(0.0) : D;
}
// eX_lsda of the vsxc module
template <int N>
DN<N> vs_ex(const DN<N>& r) {
  return r.v >= VS_DTOL ? -0.930525736349100 * dpow(r, 4.0 / 3.0) : cst<N>(0.0);
}

inline const double* vsxc_dx(int set) {  // get_pars_vsxc_exchange
  static const double p[3][6] = {
      {1.05324147599106640E+00, 3.82234242542822070E-03, -6.71698348131996321E-03, 2.53030938105796706E-05,
       1.37850244210630278E-04, -3.84172286736070984E-04},
      {6.012244E-01, 4.748822E-03, -8.635108E-03, -9.308062E-06, 4.482811E-05, 0.0},
      {1.422057E-01, 7.370319E-04, -1.601373E-02, 0.0, 0.0, 0.0}};
  return p[set];
}
inline const double* vsxc_dc(int set, int term) {  // get_pars_vsxc_correlation: term 1 same spin, 2 opposite
  static const double p[3][2][6] = {
      {{3.270912E-01, -3.228915E-02, -2.942406E-02, 2.134222E-03, -5.451559E-03, 1.577575E-02},
       {7.035010E-01, 7.694574E-03, 5.152765E-02, 3.394308E-05, -1.269420E-03, 1.296118E-03}},
      {{4.650534E-01, 1.617589E-01, 1.833657E-01, 4.692100E-04, -4.990573E-03, 0.0},
       {3.957626E-01, -5.614546E-01, 1.403963E-02, 9.831442E-04, -3.577176E-03, 0.0}},
      {{4.905945E-01, -1.437348E-01, 2.357824E-01, 1.871015E-03, -3.788963E-03, 0.0},
       {-2.741539E+00, -6.720113E-01, -7.932688E-02, 1.918681E-03, -2.032902E-03, 0.0}}};
  return p[set][term - 1];
}

// vsxc_exchange of one spin: e_x^LSDA h(x_s^2, z_s), alpha = 0.00186726
template <int N>
DN<N> vsxc_x_spin(int set, const DN<N>& r, const DN<N>& g, const DN<N>& t) {
  return vs_ex(r) * gvt4(0.00186726, vsxc_dx(set), vs_x2(r, g), vs_z(r, t));
}

// vsxc_correlation (spin-resolved input): same-spin terms e_s h_ss D_s and the
// opposite-spin term (e_c(a, b) - e_c(a, 0) - e_c(0, b)) h_os with summed
// x^2 and z.  A spin density below 1e-30 has no derivatives (the reference
// masks its derivative terms there).
template <int N>
DN<N> vsxc_c(int set, DN<N> ra, DN<N> rb, const DN<N>& gaa, const DN<N>& gbb, const DN<N>& ta, const DN<N>& tb) {
  if (!(ra.v >= VS_DTOL)) ra = cst<N>(ra.v);
  if (!(rb.v >= VS_DTOL)) rb = cst<N>(rb.v);
  const DN<N> zero = cst<N>(0.0);
  const DN<N> ea = pw92_c_lda(ra, zero), eb = pw92_c_lda(zero, rb);
  const DN<N> eo = pw92_c_lda(ra, rb) - ea - eb;
  DN<N> F = zero;
  if (ra.v >= VS_DTOL) F = F + ea * gvt4(0.00515088, vsxc_dc(set, 1), vs_x2(ra, gaa), vs_z(ra, ta)) * vs_dsic(ra, gaa, ta);
  if (rb.v >= VS_DTOL) F = F + eb * gvt4(0.00515088, vsxc_dc(set, 1), vs_x2(rb, gbb), vs_z(rb, tb)) * vs_dsic(rb, gbb, tb);
  if ((ra + rb).v >= VS_DTOL)
    F = F + eo * gvt4(0.00304966, vsxc_dc(set, 2), vs_x2(ra, gaa) + vs_x2(rb, gbb), vs_z(ra, ta) + vs_z(rb, tb));
  return F;
}

inline const double* m06_a(int set) {  // get_pars_m06_exchange, a(0:11)
  static const double p[2][12] = {
      {3.987756E-01, 2.548219E-01, 3.923994E-01, -2.103655E+00, -6.302147E+00, 1.097615E+01, 3.097273E+01,
       -2.318489E+01, -5.673480E+01, 2.160364E+01, 3.421814E+01, -9.049762E+00},
      {5.877943E-01, -1.371776E-01, 2.682367E-01, -2.515898E+00, -2.978892E+00, 8.710679E+00, 1.688195E+01,
       -4.489724E+00, -3.299983E+01, -1.449050E+01, 2.043747E+01, 1.256504E+01}};
  return p[set - 1];
}
inline const double* m06_c(int set, int term) {  // get_pars_m06_correlation
  static const double p[2][2][5] = {
      {{5.349466E-01, 5.396620E-01, -3.161217E+01, 5.149592E+01, -2.919613E+01},
       {6.042374E-01, 1.776783E+02, -2.513252E+02, 7.635173E+01, -1.255699E+01}},
      {{5.094055E-01, -1.491085E+00, 1.723922E+01, -3.859018E+01, 2.845044E+01},
       {3.741539E+00, 2.187098E+02, -4.531252E+02, 2.936479E+02, -6.287470E+01}}};
  return p[set - 1][term - 1];
}

// m06_exchange of one spin: e_x^LSDA F_PBE(x^2) f(w) (pbeef, kedef) plus vsxc_exchange of the set
template <int N>
DN<N> m06_x_spin(int set, const DN<N>& r, const DN<N>& g, const DN<N>& t) {
  const double pbec2 = 4.49267E-3, pbec1 = 3.612108584108E-03, CT = 4.55779987234560;
  const DN<N> x2 = vs_x2(r, g);
  const DN<N> pf = 1.0 + pbec1 * x2 / (1.0 + pbec2 * x2);
  DN<N> w = cst<N>(0.0);
  if (r.v >= VS_DTOL && t.v >= VS_DTOL) {
    const DN<N> tu = CT * dpow(r, 5.0 / 3.0);
    w = (tu - t) / (tu + t);
  }
  const double* a = m06_a(set);
  DN<N> k = cst<N>(a[11]);
  for (int j = 10; j >= 0; --j) k = k * w + a[j];
  return vs_ex(r) * pf * k + vsxc_x_spin(set, r, g, t);
}

// bmk_term: c0 + c1 v + ... + c4 v^4, v = beta x^2 / (1 + beta x^2)
template <int N>
DN<N> bmk(double beta, const double* c, const DN<N>& x2) {
  const DN<N> v = beta * x2 / (1.0 + beta * x2);
  return c[0] + (c[1] + (c[2] + (c[3] + c[4] * v) * v) * v) * v;
}

// m06_correlation: vsxc_correlation of the set plus the B97-type terms
template <int N>
DN<N> m06_cor(int set, const DN<N>& ra, const DN<N>& rb, const DN<N>& gaa, const DN<N>& gbb, const DN<N>& ta,
              const DN<N>& tb) {
  const DN<N> zero = cst<N>(0.0);
  const DN<N> ea = pw92_c_lda(ra, zero), eb = pw92_c_lda(zero, rb);
  const DN<N> eo = pw92_c_lda(ra, rb) - ea - eb;
  const DN<N> xa = vs_x2(ra, gaa), xb = vs_x2(rb, gbb);
  DN<N> F = vsxc_c(set, ra, rb, gaa, gbb, ta, tb);
  F = F + ea * bmk(0.06, m06_c(set, 1), xa) * vs_dsic(ra, gaa, ta);
  F = F + eb * bmk(0.06, m06_c(set, 1), xb) * vs_dsic(rb, gbb, tb);
  return F + eo * bmk(0.0031, m06_c(set, 2), xa + xb);
}

// VSXC / M06-L / M06 of the spin-resolved quantities (gamma_ab is not used)
template <int N>
DN<N> vs_family(int set, const DN<N>& ra, const DN<N>& rb, const DN<N>& gaa, const DN<N>& gbb, const DN<N>& ta,
                const DN<N>& tb) {
  if (set == 0) return vsxc_x_spin(0, ra, gaa, ta) + vsxc_x_spin(0, rb, gbb, tb) + vsxc_c(0, ra, rb, gaa, gbb, ta, tb);
  return m06_x_spin(set, ra, gaa, ta) + m06_x_spin(set, rb, gbb, tb) + m06_cor(set, ra, rb, gaa, gbb, ta, tb);
}

// A meta-GGA at one point (set: -1 TPSS, 0 VSXC, 1 M06-L, 2 M06): f and its
// derivatives in the reference's layout (ispin 1: rho, gamma, tau of the
// total density; ispin 2: rho_a, rho_b; gamma_aa, gamma_bb, gamma_ab; tau_a,
// tau_b).  The closed shell is the open form at rho/2, gamma/4, tau/2, as
// the reference's wrappers evaluate it; its derivatives are the chain rule of
// that (tpss_X, m06_X, m06_C), except that vsxc_X and vsxc_C scale the
// spin-a derivatives by 0.5, 0.25, 0.5 (vsxc_mgga_module.f90:127-131,
// :213-217), half the chain rule, which is restated as it is.
inline void mgga_point(int set, int ispin, const double* rho, const double* gam, const double* tau, double& f,
                       double* fr, double* fg, double* ft) {
  if (ispin == 1) {
    const DN<3> r = var<3>(0, rho[0]), g = var<3>(1, gam[0]), t = var<3>(2, tau[0]);
    const DN<3> hr = 0.5 * r, qg = 0.25 * g, ht = 0.5 * t;
    const DN<3> F = set < 0 ? 2.0 * tpss_x_spin(hr, qg, ht) + tpss_c(hr, hr, qg, qg, qg, ht, ht, true)
                            : vs_family(set, hr, hr, qg, qg, ht, ht);
    const double h = set == 0 ? 0.5 : 1.0;
    f = F.v;
    fr[0] = h * F.d[0];
    fg[0] = h * F.d[1];
    ft[0] = h * F.d[2];
    return;
  }
  const DN<7> ra = var<7>(0, rho[0]), rb = var<7>(1, rho[1]);
  const DN<7> gaa = var<7>(2, gam[0]), gbb = var<7>(3, gam[1]), gab = var<7>(4, gam[2]);
  const DN<7> ta = var<7>(5, tau[0]), tb = var<7>(6, tau[1]);
  const DN<7> F = set < 0 ? tpss_x_spin(ra, gaa, ta) + tpss_x_spin(rb, gbb, tb) +
                                tpss_c(ra, rb, gaa, gbb, gab, ta, tb, false)
                          : vs_family(set, ra, rb, gaa, gbb, ta, tb);
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
