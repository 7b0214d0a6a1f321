// xc_functional.cuh -- per-point XC functionals in FP64, closed-shell (ispin=1).
//
// Restates ParaGauss's functional pieces with hand-derived first derivatives
// (the reference obtains them with its forward-mode AD types):
//   Slater exchange       modules/exchange.f90:511-601  (x_lda)
//   VWN5 correlation      modules/vwnc.f90:122-297      (c_lda, vwn_ldac)
//   PW92 correlation      modules/pw_ldac_module.f90:127-312, :591-651
//   PBE exchange G(s^2)   modules/exchange.f90:325-439, :617-639, :858-867
//   PBE correlation H     modules/pbe_ggcxc_module.f90:96-348
// composed as the XC keywords do (modules/xc_cntrl.f90:460-465, :652-670):
//   "VWN" = Slater + VWN5, "PBE" = Slater + PW92 + PBE-X(G) + PBE-C(H).
// Literal constants, density guards and epsilons are the reference's.
#pragma once

#include <cmath>

namespace pgxc {

// Constants that the reference computes with library pow(); filled on the
// host (glibc) so that they round exactly as in the Fortran build.
struct XcConst {
  double xalpha;        // -(3/4)(3/pi)^(1/3)
  // VWN
  double vwn_fact;      // 3/(4 pi)
  double vwn_third;
  // PW92
  double pw_crs;        // (3/(4 pi))^(1/3)
  // PBE exchange
  double s2_fact;       // 1/(4 (3 pi^2)^(2/3))
  double pbe_mu;        // beta*pi^2/3
  // PBE correlation
  double pbe_fi;        // (0.5^(2/3)+0.5^(2/3)) * (1/2^(1/3))
  double pbe_ct;        // pi/(16 (3 pi^2)^(1/3))
};

__host__ inline XcConst make_xc_const() {
  XcConst c;
  const double pi_x = 3.14159265358979324;  // exchange.f90 uses constants.f90 pi
  c.xalpha = -(3.0 / 4.0) * std::pow(3.0 / pi_x, 1.0 / 3.0);
  const double pi_v = 3.141592653589793240;  // vwnc.f90:140
  c.vwn_fact = 3.0 / (4.0 * pi_v);
  c.vwn_third = 1.0 / 3.0;
  const double pi_p = 3.14159265358979324;   // pw_ldac_module.f90:120
  c.pw_crs = std::pow(3.0 / (4.0 * pi_p), 1.0 / 3.0);
  c.s2_fact = 1.0 / (4.0 * std::pow(3.0 * pi_x * pi_x, 2.0 / 3.0));
  c.pbe_mu = 0.066725 * (pi_x * pi_x / 3.0);
  c.pbe_fi = (std::pow(0.5, 2.0 / 3.0) + std::pow(0.5, 2.0 / 3.0)) * (1.0 / std::pow(2.0, 1.0 / 3.0));
  c.pbe_ct = pi_p / (4.0 * 4.0 * std::pow(3.0 * pi_p * pi_p, 1.0 / 3.0));
  return c;
}

// VWN interpolation ec(X; B, C, X0) of vwnc.f90:199-212 and d ec / dX.
__device__ __forceinline__ void vwn_ec(double X, double B, double C, double X0, double& e, double& de) {
  const double Q = sqrt(4.0 * C - B * B);
  const double XX0 = (X0 + B) * X0 + C;
  const double XXX = (X + B) * X + C;
  const double tX = 2.0 * X + B;
  const double FXX = atan(Q / tX);
  const double dF = -2.0 * Q / (tX * tX + Q * Q);
  const double c1 = 2.0 * B / Q;
  const double c2 = B * X0 / XX0;
  const double c3 = (2.0 * (B + 2.0 * X0)) / Q;
  const double Xm = X - X0;
  e = log(X * X / XXX) + c1 * FXX - c2 * (log(Xm * Xm / XXX) + c3 * FXX);
  de = 2.0 / X - tX / XXX + c1 * dF - c2 * (2.0 / Xm - tX / XXX + c3 * dF);
}

// PW92 G(rs) for the unpolarised (ECU) parameters, pw_ldac_module.f90:171-192
// with set_param :599-606, and its derivative in rs.
__device__ __forceinline__ void pw92_ecu(double rs, double& E, double& dE) {
  const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
  const double rs12 = sqrt(rs);
  const double Q0 = -2.0 * a * (1.0 + a1 * rs);
  const double Q1 = 2.0 * a * (b1 * rs12 + b2 * rs + b3 * rs * rs12 + b4 * rs * rs);
  const double Q2 = log(1.0 + 1.0 / Q1);
  const double dQ1 = 2.0 * a * (0.5 * b1 / rs12 + b2 + 1.5 * b3 * rs12 + 2.0 * b4 * rs);
  E = Q0 * Q2;
  dE = -2.0 * a * a1 * Q2 - Q0 * dQ1 / (Q1 * (Q1 + 1.0));
}

// Slater exchange, closed shell: x_lda with rho > 0 guard.
__device__ __forceinline__ void slater(const XcConst& K, double n, double& f, double& fr) {
  if (n > 0.0) {
    const double c = cbrt(n);
    f += K.xalpha * n * c;
    fr += (4.0 / 3.0) * K.xalpha * c;
  }
}

// "VWN": Slater + VWN5 (c_lda at na = nb = n/2, where the spin
// interpolation vanishes identically).
__device__ __forceinline__ void xc_vwn(const XcConst& K, double n, double& f, double& fr) {
  f = 0.0;
  fr = 0.0;
  slater(K, n, f, fr);
  const double ap = 0.0621841 / 2.0, bp = 3.72744, cp = 12.9352, x0p = -0.10498;
  const double S = n + 1.0e-50;                 // sums = na + nb + deps
  const double X = sqrt(pow(K.vwn_fact / S, K.vwn_third));
  double e, de;
  vwn_ec(X, bp, cp, x0p, e, de);
  const double ecpara = ap * e;
  f += ecpara * S;
  fr += ecpara - ap * de * X / 6.0;             // dX/dn = -X/(6S)
}

// "PBE": Slater + PW92 + PBE exchange enhancement + PBE correlation H.
// n = total density, g = |grad n|^2; returns f, df/dn, df/dg.
__device__ __forceinline__ void xc_pbe(const XcConst& K, double n, double g, double& f, double& fr,
                                       double& fg) {
  f = 0.0;
  fr = 0.0;
  fg = 0.0;
  // Slater (XALPHA)
  slater(K, n, f, fr);
  // PW92 at na = nb = n/2 (PWLDAC): nn = n, frozen at 1e-30 below it
  {
    const bool frozen = n < 1.0e-30;
    const double nn = frozen ? 1.0e-30 : n;
    const double rs = K.pw_crs / cbrt(nn);
    double E, dE;
    pw92_ecu(rs, E, dE);
    f += nn * E;
    if (!frozen) fr += E - rs * dE / 3.0;
  }
  // PBE exchange: e_x * G(s^2), the 1 of (1+G) omitted (x_gga)
  {
    double ex = 0.0, exr = 0.0;
    if (n > 0.0) {
      const double c = cbrt(n);
      ex = K.xalpha * n * c;
      exr = (4.0 / 3.0) * K.xalpha * c;
    }
    double s2 = 0.0, s2r = 0.0, s2g = 0.0;
    if (n >= 1.0e-20) {
      const double c = cbrt(n);
      const double n83 = n * n * c * c;
      s2g = 1.0 / n83 * K.s2_fact;
      s2 = g * s2g;
      s2r = -(8.0 / 3.0) * s2 / n;
    }
    const double kappa = 0.804, mu = K.pbe_mu;
    const double den = kappa + mu * s2;
    const double G = kappa * mu * s2 / den;
    const double Gs = kappa * kappa * mu / (den * den);
    f += ex * G;
    fr += exr * G + ex * Gs * s2r;
    fg += ex * Gs * s2g;
  }
  // PBE correlation H (c_gga with na = nb = n/2)
  if (n > 0.0) {
    const double beta = 0.066725;
    const double gam = 0.03109069086965489503494086371;
    const double deps = 1.0e-30;
    double EL, dEL;
    if (n >= 1.0e-30) {
      const double rs = K.pw_crs / cbrt(n);
      double E, dE;
      pw92_ecu(rs, E, dE);
      EL = (n * E) / n;
      dEL = dE * (-rs / (3.0 * n));
    } else {  // c_lda froze nn at deps: ELDAC = const / n
      const double rs = K.pw_crs / cbrt(1.0e-30);
      double E, dE;
      pw92_ecu(rs, E, dE);
      const double cl = 1.0e-30 * E;
      EL = cl / n;
      dEL = -cl / (n * n);
    }
    const double fi = K.pbe_fi;
    const double fi2 = fi * fi;
    const double fi3 = fi2 * fi;
    const double ge = gam * fi3;
    const double bg = beta / gam;
    const double E1 = exp(-EL / ge);
    const double aden = E1 - 1.0 + deps;
    const double A = bg / aden;
    const double dA = bg * E1 * (dEL / ge) / (aden * aden);
    const double c = cbrt(n);
    const double n73 = n * n * c;
    const double dn73 = (7.0 / 3.0) * n * c;
    const double tden = fi2 * n73 + deps;
    const double t2 = g / tden * K.pbe_ct;
    const double dt2n = -g * K.pbe_ct * fi2 * dn73 / (tden * tden);
    const double dt2g = K.pbe_ct / tden;
    const double x = A * t2;
    const double dxn = dA * t2 + A * dt2n;
    const double dxg = A * dt2g;
    const double rden = 1.0 + x + x * x;
    const double rat = (1.0 + x) / rden;
    const double drat = -x * (2.0 + x) / (rden * rden);
    const double u = bg * t2 * rat;
    const double dun = bg * (dt2n * rat + t2 * drat * dxn);
    const double dug = bg * (dt2g * rat + t2 * drat * dxg);
    const double H = ge * log(1.0 + u);
    const double dHn = ge * dun / (1.0 + u);
    const double dHg = ge * dug / (1.0 + u);
    f += n * H;
    fr += H + n * dHn;
    fg += n * dHg;
  }
}

}  // namespace pgxc
