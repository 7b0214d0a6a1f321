// xc_functional.cuh -- per-point XC functionals in FP64.
//
// Closed shell (ispin = 1) with hand-derived first derivatives; open shell
// (ispin = 2) with forward-mode dual numbers in (rho_a, rho_b, gamma), the
// role of the reference's ad2x1..ad2x3 types (autodiff/autodiff2.f90).
// Restated pieces:
//   Slater exchange       modules/exchange.f90:511-601  (x_lda)
//   VWN5 correlation      modules/vwnc.f90:122-297      (c_lda, vwn_ldac)
//   PW92 correlation      modules/pw_ldac_module.f90:127-312, :591-651
//   PBE exchange G(s^2)   modules/exchange.f90:325-439, :617-639, :858-867
//   PBE correlation H     modules/pbe_ggcxc_module.f90:96-348
//   Becke 88 G(s^2)       modules/exchange.f90:672-705, :964-991
//   PW91 exchange G(s^2)  modules/exchange.f90:919-962
//   PBEN, VMT, VT84 G(s^2) modules/exchange.f90:723-856, :869-902
//   Perdew 86 correlation modules/becke_perdew_module.f90:125-260
//   PW91 correlation      modules/gga_response_module.f90:278-918 (H0 + H1)
//   LYP correlation       modules/lyp.f90 (lyp_C, lyp_corr)
//   HCTH                  modules/hcth.f90 (pg_hcth, hcth_x_calc, hcth_c_calc)
// composed as the XC keywords do (modules/xc_cntrl.f90:460-798):
//   "VWN" = Slater + VWN5, "PBE" = Slater + PW92 + PBE-X(G) + PBE-C(H),
//   "BP" = Slater + VWN5 + B88 + P86, "PW91" = Slater + PW92 + PW91-X + PW91-C,
//   "BPW91" = Slater + PW92 + B88 + PW91-C, "BLYP" = Slater + B88 + LYP,
//   "XALPHA" = Slater, "B88" = Slater + B88, "PBEN" / "VMT" / "VT84" /
//   "VMTsol" / "VT84sol" = Slater + PW92 + their G + PBE-C, "HCTH*" = HCTH
//   exchange + correlation alone, "NRECMV92" = Slater + ECMV92 G, "PWLDA" =
//   Slater + PW92 (an LDA); the hybrids' grid parts "B3LYP" and "PBE0" weight
//   the pieces by their fractions (the exact exchange is not a grid term).
// Literal constants, density guards and epsilons are the reference's.
#pragma once

#include <cmath>

#include "../../include/pgxc.h"

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
  double pbe_kappa;     // enhancement-factor kappa (PBE 0.804, revPBE 1.245)
  double pbe_mu;        // beta*pi^2/3 (PBE, revPBE) or 10/81 (PBEsol)
  double pbe_beta;      // correlation beta (PBE 0.066725, PBEsol 0.046)
  // Becke 88: exchange enhancement constants of g_becke88
  double b88_A, b88_B, b88_D;
  // LYP: 2^(11/3)
  double lyp_2113;
  double vmt_alpha;     // alpha of the VMT / VT84 enhancements
  int xg;               // exchange enhancement G(s^2): XG_*
  int cg;               // gradient correlation: CG_*
  int lc;               // LDA correlation: LC_VWN, LC_PW92 or LC_NONE
  // fractions of the pieces (xc_cntrl frac, applied as xc_functionals does,
  // xc_func.f90:284-305): Slater, exchange enhancement, LDA correlation,
  // gradient correlation; 1 except in the hybrids' grid parts
  double fx_lda, fx_g, fc_lda, fc_g;
  int lb94;             // 1: add the LB94 potential correction ("LB94")
  double lb94_two13;    // 2^(1/3)
  // relativistic exchange (exchange.f90 x_lda / x_gga with X_LONGTRANS):
  // rel_lda: Slater times phi0(beta) ("RVWN"); rel_g: the enhancement term
  // e_x (phi0 - 1 + phi2 G) with the Pade set of Becke 88 (1, "RBP") or of
  // ECMV92 (2, "ECMV92"); rvwn: add ec_RLDA (1, relxc.f90) or VWN5 (phic0 - 1)
  // (2, "RVWN:Engel", exchange.f90 correlation_lda); rel_c: speed of light
  int rel_lda, rel_g, rvwn;
  double rel_c, rel_3pi2;
  // rpw91c: "RPW91" adds phi_c(n) times the H of pw91c_calc (relxc.f90:162-218)
  int rpw91c;
  // PBE correlation
  double pbe_fi;        // (0.5^(2/3)+0.5^(2/3)) * (1/2^(1/3))
  double pbe_ct;        // pi/(16 (3 pi^2)^(1/3))
  // open shell
  double vwn_ffact;     // (1/2) / (2^(1/3) - 1)
  double pw_cf;         // 1 / (2^(4/3) - 2)
  double pbe_two13i;    // 1 / 2^(1/3)
  // HCTH: version 1..4 (0: not HCTH), its power-series coefficients of
  // exchange, same-spin and opposite-spin correlation, and the spin-resolved
  // Slater constant -(3/2)(3/(4 pi))^(1/3)
  int hcth;
  double hcth_x[5], hcth_caa[5], hcth_cab[5];
  double hcth_xa;
};

// HCTH coefficients c_0..c_4 of exchange, same-spin and opposite-spin
// correlation for versions 1..4 (HCTH/93, /120, /147, /407), as tabulated in
// modules/hcth.f90:80-150 (the published sets).
constexpr double kHcth[4][3][5] = {
    {{1.09320, -0.744056, 5.59920, -6.78549, 4.49357},
     {0.222601, -0.0338622, -0.0125170, -0.802496, 1.55396},
     {0.729974, 3.35287, -11.5430, 8.08564, -4.47857}},
    {{1.09163, -0.747215, 5.07833, -4.10746, 1.17173},
     {0.489508, -0.260699, 0.432917, -1.99247, 2.48531},
     {0.514730, 6.92982, -24.7073, 23.1098, -11.3234}},
    {{1.09025, -0.799194, 5.57212, -5.86760, 3.04544},
     {0.562576, 0.0171436, -1.30636, 1.05747, 0.885429},
     {0.542352, 7.01464, -28.3822, 35.0329, -20.4284}},
    {{1.08184, -0.518339, 3.42562, -2.62901, 2.28855},
     {1.18777, -2.40292, 5.61741, -9.17923, 6.24798},
     {0.589076, 4.42374, -19.2218, 42.5721, -42.0052}}};

// GGA pieces of a keyword.  Exchange enhancement: the PBE form (kappa, mu),
// Becke 88, or PW91.  Correlation: PW92 + PBE H, VWN5 + Perdew 86, PW92 +
// PW91 H0 + H1, or LYP (a whole correlation: no LDA part).
constexpr int XG_PBE = 0, XG_B88 = 1, XG_PW91 = 2, XG_PBEN = 3, XG_VMT = 4, XG_VT84 = 5, XG_ECMV92 = 6, XG_NONE = 7;
constexpr int CG_PBE = 0, CG_P86 = 1, CG_PW91 = 2, CG_LYP = 3, CG_NONE = 4;
constexpr int LC_VWN = 0, LC_PW92 = 1, LC_NONE = 2;

// Constants of the functional (PGXC_XC_*): the PBE-form keywords differ only
// in their parameters (exchange.f90 g_pbe / g_revpbe / g_pbesol :617-670,
// pbe_ggcxc_module.f90 pbe_ggcc :249-270), the others in their pieces.
__host__ inline XcConst make_xc_const(int functional = PGXC_XC_PBE) {
  XcConst c;
  const double pi_x = 3.14159265358979324;  // exchange.f90 uses constants.f90 pi
  c.xalpha = -(3.0 / 4.0) * std::pow(3.0 / pi_x, 1.0 / 3.0);
  const double pi_v = 3.141592653589793240;  // vwnc.f90:140
  c.vwn_fact = 3.0 / (4.0 * pi_v);
  c.vwn_third = 1.0 / 3.0;
  const double pi_p = 3.14159265358979324;   // pw_ldac_module.f90:120
  c.pw_crs = std::pow(3.0 / (4.0 * pi_p), 1.0 / 3.0);
  c.s2_fact = 1.0 / (4.0 * std::pow(3.0 * pi_x * pi_x, 2.0 / 3.0));
  c.pbe_kappa = functional == PGXC_XC_REVPBE ? 1.245 : 0.804;
  const bool sol = functional == PGXC_XC_PBESOL || functional == PGXC_XC_VMTSOL || functional == PGXC_XC_VT84SOL;
  c.pbe_mu = sol ? 10.0 / 81.0 : 0.066725 * (pi_x * pi_x / 3.0);
  c.pbe_beta = functional == PGXC_XC_PBESOL ? 0.046 : 0.066725;
  // g_becke88, exchange.f90:672-705 (BECKE88_0042: beta = 0.0042)
  c.b88_A = 6.0 * 0.0042 * std::pow(2.0, 1.0 / 3.0) * std::pow(3.0 * pi_x * pi_x, 1.0 / 3.0) * 2.0;
  c.b88_D = c.b88_A * (4.0 * pi_x) / 9.0;
  c.b88_B = 2.0 * std::pow(6.0 * pi_x * pi_x, 1.0 / 3.0);
  c.lyp_2113 = std::pow(2.0, 11.0 / 3.0);
  // g_vmt :723-737, g_vt84 :739-760, g_vmtsol :762-775, g_vt84sol :777-797
  c.vmt_alpha = functional == PGXC_XC_VMT ? 0.002762 : functional == PGXC_XC_VT84 ? 0.000069
                : functional == PGXC_XC_VMTSOL ? 0.0015532 : functional == PGXC_XC_VT84SOL ? 0.000023 : 0.0;
  const int f = functional;
  const bool b88 =
      f == PGXC_XC_BP86 || f == PGXC_XC_BPW91 || f == PGXC_XC_BLYP || f == PGXC_XC_B88 || f == PGXC_XC_B3LYP;
  const bool ecmv = f == PGXC_XC_NRECMV92;
  c.xg = b88 ? XG_B88
         : ecmv ? XG_ECMV92
         : f == PGXC_XC_PW91 ? XG_PW91
         : f == PGXC_XC_PBEN ? XG_PBEN
         : (f == PGXC_XC_VMT || f == PGXC_XC_VMTSOL) ? XG_VMT
         : (f == PGXC_XC_VT84 || f == PGXC_XC_VT84SOL) ? XG_VT84 : XG_PBE;
  c.cg = f == PGXC_XC_BP86 ? CG_P86
         : (f == PGXC_XC_PW91 || f == PGXC_XC_BPW91) ? CG_PW91
         : (f == PGXC_XC_BLYP || f == PGXC_XC_B3LYP) ? CG_LYP
         : (f == PGXC_XC_B88 || ecmv || !PGXC_XC_IS_GGA(f)) ? CG_NONE : CG_PBE;
  c.lc = (f == PGXC_XC_VWN || f == PGXC_XC_BP86 || f == PGXC_XC_B3LYP) ? LC_VWN
         : (f == PGXC_XC_XALPHA || f == PGXC_XC_B88 || f == PGXC_XC_BLYP || ecmv) ? LC_NONE : LC_PW92;
  c.fx_lda = c.fx_g = c.fc_lda = c.fc_g = 1.0;
  c.lb94 = f == PGXC_XC_LB94 ? 1 : 0;
  c.lb94_two13 = std::pow(2.0, 1.0 / 3.0);
  c.rel_c = 137.03604;  // constants.f90 SPEED_OF_LIGHT
  c.rel_3pi2 = 3.0 * 3.14159265358979324 * 3.14159265358979324;
  c.rel_lda = (f == PGXC_XC_RVWN || f == PGXC_XC_RVWN_ENGEL) ? 1 : 0;
  c.rvwn = f == PGXC_XC_RVWN ? 1 : f == PGXC_XC_RVWN_ENGEL ? 2 : 0;
  c.rel_g = (f == PGXC_XC_RBP || f == PGXC_XC_RPW91) ? 1 : f == PGXC_XC_ECMV92 ? 2 : 0;
  c.rpw91c = f == PGXC_XC_RPW91 ? 1 : 0;
  if (f == PGXC_XC_RVWN || f == PGXC_XC_RVWN_ENGEL) {
    // "RVWN": RXAlpha + VWN + rel_vwn_calc, "RVWN:Engel": correlation_lda (xc_cntrl.f90:477-498)
    c.lc = LC_VWN;
    c.cg = CG_NONE;
  } else if (f == PGXC_XC_RBP) {  // "RBP": XAlpha + VWN + RBecke88 + Perdew (:545-558)
    c.xg = XG_B88;
    c.cg = CG_P86;
    c.lc = LC_VWN;
  } else if (f == PGXC_XC_RPW91) {  // "RPW91": PW92 + RPW91x (no XAlpha) + PW91c + RPW91c (:626-636)
    c.xg = XG_PW91;
    c.cg = CG_PW91;
    c.lc = LC_PW92;
    c.fx_lda = 0.0;
  } else if (f == PGXC_XC_ECMV92) {  // "ECMV92": XAlpha + ECMV92 with X_LONGTRANS (:645-650)
    c.xg = XG_ECMV92;
    c.cg = CG_NONE;
    c.lc = LC_NONE;
  }
  if (c.lb94) {  // "LB94": XAlpha + VWN + baerends94 (a potential term only)
    c.xg = XG_NONE;
    c.cg = CG_NONE;
    c.lc = LC_VWN;
  }
  if (f == PGXC_XC_B3LYP) {  // "B3LYP" (xc_cntrl.f90:965-985): 0.80 XAlpha, 0.72 B88, 0.19 VWN, 0.81 LYP
    c.fx_lda = 0.80;
    c.fx_g = 0.72;
    c.fc_lda = 0.19;
    c.fc_g = 0.81;
  } else if (f == PGXC_XC_PBE0) {  // "PBE0" (:996-1016): 0.75 XAlpha, 0.75 PBE-X, PW92, PBE-C
    c.fx_lda = 0.75;
    c.fx_g = 0.75;
  }
  c.hcth = (f >= PGXC_XC_HCTH && f <= PGXC_XC_HCTH407) ? f - PGXC_XC_HCTH + 1 : 0;
  for (int n = 0; n < 5; ++n) {
    const int v = c.hcth > 0 ? c.hcth - 1 : 0;
    c.hcth_x[n] = kHcth[v][0][n];
    c.hcth_caa[n] = kHcth[v][1][n];
    c.hcth_cab[n] = kHcth[v][2][n];
  }
  c.hcth_xa = -(3.0 / 2.0) * std::pow(3.0 / (4.0 * 3.14159265358979324), 1.0 / 3.0);
  c.pbe_fi = (std::pow(0.5, 2.0 / 3.0) + std::pow(0.5, 2.0 / 3.0)) * (1.0 / std::pow(2.0, 1.0 / 3.0));
  c.pbe_ct = pi_p / (4.0 * 4.0 * std::pow(3.0 * pi_p * pi_p, 1.0 / 3.0));
  c.vwn_ffact = 0.5 / (std::pow(2.0, 1.0 / 3.0) - 1.0);
  c.pw_cf = 1.0 / (std::pow(2.0, 4.0 / 3.0) - 2.0);
  c.pbe_two13i = 1.0 / std::pow(2.0, 1.0 / 3.0);
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

// Relativistic beta = (3 pi^2 n)^(1/3) / c (rbeta, exchange.f90:993-1005; 0 below
// n = 1e-20) and d beta / dn.
__device__ __forceinline__ void rel_beta(const XcConst& K, double n, double& b, double& db) {
  if (n >= 1.0e-20) {
    b = pow(K.rel_3pi2 * n, 1.0 / 3.0) / K.rel_c;
    db = b / (3.0 * n);
  } else {
    b = 0.0;
    db = 0.0;
  }
}

// phi0 for X_LONGTRANS: 1 - (3/2) t4^2, t4 = (eta - arcsinh(b)/b)/b,
// eta = sqrt(1 + b^2), its series 2b/3 - b^3/5 + 3b^5/28 below |b| = 1e-4, and 0
// at b = 0 (phi0, exchange.f90:1008-1098); d phi0 / db.
__device__ __forceinline__ void rel_phi0(double b, double& phi, double& dphi) {
  if (b == 0.0) {
    phi = 0.0;
    dphi = 0.0;
    return;
  }
  double t4, dt4;
  if (fabs(b) > 1.0e-4) {
    const double eta = sqrt(1.0 + b * b);
    const double ash = log(b + eta);  // arcsinh, autodiff2.f90:791-820 (|b| >= 1e-4)
    t4 = (eta - ash / b) / b;
    dt4 = -2.0 / (eta * b * b) + 2.0 * ash / (b * b * b);
  } else {
    const double b2 = b * b, b4 = b2 * b2;
    t4 = (2.0 / 3.0) * b + (-(1.0 / 5.0) * b * b2) + (3.0 / 28.0) * b * b4;
    dt4 = 2.0 / 3.0 - (3.0 / 5.0) * b2 + (15.0 / 28.0) * b4;
  }
  phi = 1.0 - 1.5 * t4 * t4;
  dphi = -3.0 * t4 * dt4;
}

// phi2 for X_LONGTRANS: the longitudinal plus the transverse 2/2 Pade in b^2,
// the RB88 set (set 1) or the RECMV92 set (set 2) (phi2 and pade22,
// exchange.f90:1100-1159); d phi2 / db.
__device__ __forceinline__ void rel_phi2(int set, double b, double& phi, double& dphi) {
  const double aL1 = set == 1 ? 2.20848 : 2.21259, aL2 = set == 1 ? 0.668684 : 0.669152;
  const double bL1 = set == 1 ? 1.33075 : 1.32998, bL2 = set == 1 ? 0.795105 : 0.794803;
  const double aT1 = set == 1 ? 3.48638 : 3.48754, aT2 = set == 1 ? 0.614753 : 0.218599;
  const double bT1 = set == 1 ? 1.32260 : 1.15417, bT2 = set == 1 ? 0.101805 : 0.015802;
  const double x = b * b;
  const double nL = 1.0 + x * (aL1 + x * aL2), dL = 1.0 + x * (bL1 + x * bL2);
  const double nT = 0.0 + x * (aT1 + x * aT2), dT = 1.0 + x * (bT1 + x * bT2);
  phi = nL / dL + nT / dT;
  const double dnL = aL1 + 2.0 * aL2 * x, ddL = bL1 + 2.0 * bL2 * x;
  const double dnT = aT1 + 2.0 * aT2 * x, ddT = bT1 + 2.0 * bT2 * x;
  dphi = ((dnL * dL - nL * ddL) / (dL * dL) + (dnT * dT - nT * ddT) / (dT * dT)) * 2.0 * b;
}

// Slater exchange, closed shell: x_lda with rho > 0 guard, times phi0(beta)
// when relativistic (K.rel_lda), times K.fx_lda.
__device__ __forceinline__ void slater(const XcConst& K, double n, double& f, double& fr) {
  if (n > 0.0) {
    const double c = cbrt(n);
    double e = K.xalpha * n * c, de = (4.0 / 3.0) * K.xalpha * c;
    if (K.rel_lda) {
      double b, db, ph, dph;
      rel_beta(K, n, b, db);
      rel_phi0(b, ph, dph);
      de = de * ph + e * dph * db;
      e = e * ph;
    }
    f += K.fx_lda * e;
    fr += K.fx_lda * de;
  }
}

// phic0(beta) of the relativistic LDA correlation of Schmid, Engel, Dreizler,
// Blaha and Schwarz (phic0, exchange.f90:159-204): (1 + a1 b^3 ln b + a2 b^4 +
// a3 (1 + b^2)^2 b^4) / (1 + b1 b^3 ln b + b2 b^4 + b3 (AA ln b + BB) b^7),
// AA = 0.0621841, BB = AA ln c + 0.05275877384; 1 at beta = 0 (n below 1e-20);
// and d phic0 / dn.
__device__ __forceinline__ void engel_phic0(const XcConst& K, double n, double& phi, double& dphi) {
  double b, db;
  rel_beta(K, n, b, db);
  if (!(b > 0.0)) {
    phi = 1.0;
    dphi = 0.0;
    return;
  }
  const double a1 = -2.44968, a2 = 1.91853, a3 = 0.0718854, b1 = -1.59583, b2 = 1.29176, b3 = 0.364044;
  const double AA = 0.0621841, BB = AA * log(K.rel_c) + 0.05275877384;
  const double bb = b * b, bbb = bb * b, b4 = bb * bb, b6 = b4 * bb, L = log(b), q = 1.0 + bb;
  const double num = 1.0 + a1 * bbb * L + a2 * b4 + a3 * q * q * b4;
  const double den = 1.0 + b1 * bbb * L + b2 * b4 + b3 * (AA * L + BB) * b6 * b;
  const double dnum = a1 * (3.0 * bb * L + bb) + 4.0 * a2 * bbb + a3 * (4.0 * b * q * b4 + 4.0 * q * q * bbb);
  const double dden = b1 * (3.0 * bb * L + bb) + 4.0 * b2 * bbb + b3 * (AA * b6 + 7.0 * (AA * L + BB) * b6);
  phi = num / den;
  dphi = (dnum * den - num * dden) / (den * den) * db;
}

// Relativistic LDA correlation correction ec_RLDA(n) and its n derivative
// (relxc.f90:221-283, the 0.25 cutoff form); 0 below n = 1e-7.  It is added to
// the energy density as it stands.
__device__ __forceinline__ void rel_vwn(const XcConst& K, double n, double& e, double& de) {
  e = 0.0;
  de = 0.0;
  if (n < 1.0e-7) return;
  const double a0 = -0.16797, b0 = 0.149530, c0 = -0.007568, d0 = 0.0504295, c1 = -0.007217, c2 = 0.0064572,
               c3 = -0.005352, d1 = 0.0995769, d2 = 0.110576, d3 = 0.0136740, d4 = 0.0311479;
  const double AA = -0.2670592864, BB = 0.5321072256;
  const double b = pow(K.rel_3pi2 * n, 1.0 / 3.0) / K.rel_c;
  if (b < 0.25) {
    e = AA * b * b * b + BB * b * b * b * b;
    de = (3.0 * AA * b * b + 4.0 * BB * b * b * b) * b / (3.0 * n);
  } else {
    const double num = c3 * b * b * b + c2 * b * b + c1 * b + c0;
    const double den = d4 * b * b * b * b + d3 * b * b * b + d2 * b * b + d1 * b + d0;
    const double dnum = 3.0 * c3 * b * b + 2.0 * c2 * b + c1;
    const double dden = 4.0 * d4 * b * b * b + 3.0 * d3 * b * b + 2.0 * d2 * b + d1;
    e = a0 * b + b0 + num / den;
    de = (a0 + (den * dnum - num * dden) / (den * den)) * b / (3.0 * n);
  }
}

// The LDA keywords, closed shell: "VWN" = Slater + VWN5 (c_lda at na = nb =
// n/2, where the spin interpolation vanishes identically), "XALPHA" (K.lc ==
// LC_NONE) = Slater, "PWLDA" (K.lc == LC_PW92) = Slater + PW92.
__device__ __forceinline__ void xc_vwn(const XcConst& K, double n, double& f, double& fr) {
  f = 0.0;
  fr = 0.0;
  slater(K, n, f, fr);
  if (K.lc == LC_NONE) return;
  if (K.lc == LC_PW92) {  // pw_ldac at na = nb = n/2: nn = n, frozen at 1e-30 below it
    const bool frozen = n < 1.0e-30;
    const double nn = frozen ? 1.0e-30 : n;
    const double rs = K.pw_crs / cbrt(nn);
    double E, dE;
    pw92_ecu(rs, E, dE);
    f += K.fc_lda * (nn * E);
    if (!frozen) fr += K.fc_lda * (E - rs * dE / 3.0);
    return;
  }
  const double ap = 0.0621841 / 2.0, bp = 3.72744, cp = 12.9352, x0p = -0.10498;
  const double S = n + 1.0e-50;                 // sums = na + nb + deps
  const double X = sqrt(pow(K.vwn_fact / S, K.vwn_third));
  double e, de;
  vwn_ec(X, bp, cp, x0p, e, de);
  const double ecpara = ap * e;
  f += K.fc_lda * (ecpara * S);
  fr += K.fc_lda * (ecpara - ap * de * X / 6.0);   // dX/dn = -X/(6S)
  if (K.rvwn == 1) {  // rel_vwn_calc (relxc.f90:128-160)
    double er, der;
    rel_vwn(K, n, er, der);
    f += er;
    fr += der;
  } else if (K.rvwn == 2) {  // correlation_lda: F (phic0 - 1), F = VWN5 of n
    double p, dp;
    engel_phic0(K, n, p, dp);
    const double F = ecpara * S;
    f += F * (p - 1.0);
    fr += (ecpara - ap * de * X / 6.0) * (p - 1.0) + F * dp;
  }
}

// GGA exchange enhancement of the closed-shell functional e(n, g): e_x G(s^2),
// the 1 of (1+G) omitted (x_gga, exchange.f90:325-439), G of the PBE form,
// of Becke 88, PW91, PBEN, VMT or VT84; adds F, dF/dn, dF/dg.
__device__ __forceinline__ void pbe_x(const XcConst& K, double n, double g, double& f, double& fr, double& fg) {
  if (K.xg == XG_NONE) return;
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
  double G, Gs;  // G(s^2) and dG/ds^2
  if (K.xg == XG_B88) {
    // Becke 88: G = D s^2 / (1 + A s asinh(B s)), below s^2 = 1e-4 its series
    // D s^2 - B A D s^4 (g_becke88_form, exchange.f90:964-991)
    const double A = K.b88_A, B = K.b88_B, Dd = K.b88_D;
    if (s2 > 1.0e-4) {
      const double s = sqrt(s2), bs = B * s, ash = asinh(bs);
      const double den = 1.0 + A * s * ash;
      // d(A s asinh(B s))/ds^2 = A (asinh(B s) + B s / sqrt(1 + B^2 s^2)) / (2 s)
      const double dden = A * (ash + bs / sqrt(1.0 + bs * bs)) / (2.0 * s);
      G = Dd * s2 / den;
      Gs = Dd / den - Dd * s2 * dden / (den * den);
    } else {
      G = s2 * (Dd - B * A * Dd * s2);
      Gs = Dd - 2.0 * B * A * Dd * s2;
    }
  } else if (K.xg == XG_PW91) {
    // PW91: G = s^2 (D - C s^2 - E exp(-100 s^2)) / (1 + A s asinh(B s) + C s^4),
    // below s^2 = 1e-4 the series s^2 (T1 + T2 s^2) (g_pw91, exchange.f90:919-962)
    const double A = 0.19645, B = 7.7956, C = 0.004, Dd = 0.2743, E = 0.1508;
    const double T1 = Dd - E, T2 = (B * A + 100.0) * E - B * A * Dd - C;
    if (s2 > 1.0e-4) {
      const double ee = E * exp(-100.0 * s2);
      const double num = Dd - C * s2 - ee;
      const double dnum = -C + 100.0 * ee;
      const double s = sqrt(s2), bs = B * s, ash = asinh(bs);
      const double den = 1.0 + A * s * ash + C * s2 * s2;
      const double dden = A * (ash + bs / sqrt(1.0 + bs * bs)) / (2.0 * s) + 2.0 * C * s2;
      G = s2 * num / den;
      Gs = (num + s2 * dnum) / den - s2 * num * dden / (den * den);
    } else {
      G = s2 * (T1 + s2 * T2);
      Gs = T1 + 2.0 * T2 * s2;
    }
  } else if (K.xg == XG_ECMV92) {
    // ECMV92: the 2/2 Pade (0.3402 s^2 + 5.9955 s^4) / (1 + 27.5026 s^2 + 5.7728 s^4)
    // (g_ecmv92 with pade22, exchange.f90:904-917, :1144-1159)
    const double a1 = 0.3402, a2 = 5.9955, b1 = 27.5026, b2 = 5.7728;
    const double num = s2 * (a1 + s2 * a2);
    const double den = 1.0 + s2 * (b1 + s2 * b2);
    G = num / den;
    Gs = ((a1 + 2.0 * a2 * s2) * den - num * (b1 + 2.0 * b2 * s2)) / (den * den);
  } else if (K.xg == XG_PBEN) {
    // PBEN: G = kappa (1 - exp(-x)), x = mu s^2 / kappa; below x = 1e-4 its
    // series to x^5 (g_pben, exchange.f90:869-902)
    const double kappa = K.pbe_kappa, mu = K.pbe_mu;
    const double x = mu * s2 / kappa;
    if (x > 1.0e-4) {
      const double e = exp(-x);
      G = kappa * (1.0 - e);
      Gs = mu * e;
    } else {
      G = kappa * x * (1.0 + x * (-1.0 / 2.0 + x * (1.0 / 6.0 + x * (-1.0 / 24.0 + x * (1.0 / 120.0)))));
      Gs = mu * (1.0 + x * (-1.0 + x * (1.0 / 2.0 + x * (-1.0 / 6.0 + x * (1.0 / 24.0)))));
    }
  } else if (K.xg == XG_VMT || K.xg == XG_VT84) {
    // VMT form mu s^2 exp(-alpha s^2) / (mu s^2 + 1) (g_vmt_form :799-817);
    // VT84 adds (1 - exp(-alpha s^4)) (1/s^2 - 1), below s^2 = 1e-4 its
    // series (g_vt84_2nd_term :819-856)
    const double mu = K.pbe_mu, a = K.vmt_alpha;
    const double e = exp(-a * s2);
    const double d = mu * s2 + 1.0;
    G = mu * s2 * e / d;
    Gs = mu * e * ((1.0 - a * s2) * d - mu * s2) / (d * d);
    if (K.xg == XG_VT84) {
      if (s2 > 1.0e-4) {
        const double e4 = exp(-a * s2 * s2);
        G += (1.0 - e4) * (1.0 / s2 - 1.0);
        Gs += 2.0 * a * s2 * e4 * (1.0 / s2 - 1.0) - (1.0 - e4) / (s2 * s2);
      } else {
        G += a * s2 * (1.0 + s2 * (-1.0 + s2 * (-a / 2.0 + s2 * (a / 2.0 + s2 * (a * a / 6.0)))));
        Gs += a * (1.0 + s2 * (-2.0 + s2 * (-1.5 * a + s2 * (2.0 * a + s2 * (5.0 * a * a / 6.0)))));
      }
    }
  } else {
    const double kappa = K.pbe_kappa, mu = K.pbe_mu;
    const double den = kappa + mu * s2;
    G = kappa * mu * s2 / den;
    Gs = kappa * kappa * mu / (den * den);
  }
  if (K.rel_g) {
    // x_gga with relativity (exchange.f90:418-438): e_x (phi0 - 1 + phi2 G), the
    // -1 for the XAlpha term (which "RPW91" leaves off all the same)
    double b, db, p0, dp0, p2, dp2;
    rel_beta(K, n, b, db);
    rel_phi0(b, p0, dp0);
    rel_phi2(K.rel_g, b, p2, dp2);
    const double fac = p0 - 1.0 + p2 * G;
    f += K.fx_g * (ex * fac);
    fr += K.fx_g * (exr * fac + ex * ((dp0 + dp2 * G) * db + p2 * Gs * s2r));
    fg += K.fx_g * (ex * p2 * Gs * s2g);
    return;
  }
  f += K.fx_g * (ex * G);
  fr += K.fx_g * (exr * G + ex * Gs * s2r);
  fg += K.fx_g * (ex * Gs * s2g);
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
    f += K.fc_lda * (nn * E);
    if (!frozen) fr += K.fc_lda * (E - rs * dE / 3.0);
  }
  // PBE exchange: e_x * G(s^2), the 1 of (1+G) omitted (x_gga)
  pbe_x(K, n, g, f, fr, fg);
  // PBE correlation H (c_gga with na = nb = n/2)
  if (n > 0.0) {
    const double beta = K.pbe_beta;
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
    f += K.fc_g * (n * H);
    fr += K.fc_g * (H + n * dHn);
    fg += K.fc_g * (n * dHg);
  }
}

// ---------------------------------------------------------------------------
// Open shell (ispin = 2).  D3 carries a value and its derivatives with
// respect to three independent inputs; the spin-resolved correlation pieces
// are written once on D3, exchange reuses the closed-shell forms through the
// spin scaling e_x[rho_a, rho_b] = (e_x[2 rho_a] + e_x[2 rho_b]) / 2.
// ---------------------------------------------------------------------------
struct D3 {
  double v, d[3];
};
__device__ __forceinline__ D3 d3c(double x) { return D3{x, {0.0, 0.0, 0.0}}; }
__device__ __forceinline__ D3 d3v(int i, double x) {
  D3 r = d3c(x);
  r.d[i] = 1.0;
  return r;
}
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}}; }
__device__ __forceinline__ D3 operator-(D3 a) { return D3{-a.v, {-a.d[0], -a.d[1], -a.d[2]}}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) {
  return D3{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
__device__ __forceinline__ D3 operator/(D3 a, D3 b) {
  const double q = b.v * b.v;
  return D3{a.v / b.v,
            {(a.d[0] * b.v - a.v * b.d[0]) / q, (a.d[1] * b.v - a.v * b.d[1]) / q, (a.d[2] * b.v - a.v * b.d[2]) / q}};
}
__device__ __forceinline__ D3 operator+(D3 a, double b) { a.v += b; return a; }
__device__ __forceinline__ D3 operator+(double b, D3 a) { a.v += b; return a; }
__device__ __forceinline__ D3 operator-(D3 a, double b) { a.v -= b; return a; }
__device__ __forceinline__ D3 operator-(double b, D3 a) { return d3c(b) - a; }
__device__ __forceinline__ D3 operator*(D3 a, double b) { return D3{a.v * b, {a.d[0] * b, a.d[1] * b, a.d[2] * b}}; }
__device__ __forceinline__ D3 operator*(double b, D3 a) { return a * b; }
__device__ __forceinline__ D3 operator/(D3 a, double b) { return D3{a.v / b, {a.d[0] / b, a.d[1] / b, a.d[2] / b}}; }
__device__ __forceinline__ D3 operator/(double b, D3 a) { return d3c(b) / a; }
// chain rule with f(a.v) and f'(a.v)
__device__ __forceinline__ D3 d3f(D3 a, double f, double df) {
  return D3{f, {df * a.d[0], df * a.d[1], df * a.d[2]}};
}
__device__ __forceinline__ D3 d3pow(D3 a, double p) { return d3f(a, pow(a.v, p), p * pow(a.v, p - 1.0)); }
__device__ __forceinline__ D3 d3sqrt(D3 a) { const double r = sqrt(a.v); return d3f(a, r, 0.5 / r); }
__device__ __forceinline__ D3 d3log(D3 a) { return d3f(a, log(a.v), 1.0 / a.v); }
__device__ __forceinline__ D3 d3exp(D3 a) { const double e = exp(a.v); return d3f(a, e, e); }
__device__ __forceinline__ D3 d3atan(D3 a) { return d3f(a, atan(a.v), 1.0 / (1.0 + a.v * a.v)); }

// VWN interpolation ec(X; B, C, X0), vwnc.f90:199-212
__device__ __forceinline__ D3 vwn_ec3(D3 X, double B, double C, double X0) {
  const double Q = sqrt(4.0 * C - B * B);
  const double XX0 = (X0 + B) * X0 + C;
  const D3 XXX = (X + B) * X + C;
  const D3 FXX = d3atan(Q / (2.0 * X + B));
  const D3 Xm = X - X0;
  return d3log(X * X / XXX) + (2.0 * B / Q) * FXX -
         (B * X0 / XX0) * (d3log(Xm * Xm / XXX) + ((2.0 * (B + 2.0 * X0)) / Q) * FXX);
}

// VWN5 c_lda(na, nb) with the spin interpolation, vwnc.f90:160-223: n * eps_c
__device__ __forceinline__ D3 vwn_c_lda(const XcConst& K, D3 na, D3 nb) {
  const double aa = -0.0337740 / 2.0, ba = 1.13107, ca = 13.0045, x0a = -0.0047584;
  const double af = 0.0310907 / 2.0, bf = 7.06042, cf = 18.0578, x0f = -0.32500;
  const double ap = 0.0621841 / 2.0, bp = 3.72744, cp = 12.9352, x0p = -0.10498;
  const double ffact = K.vwn_ffact;
  const double dfact = (4.0 / 3.0) * ffact;
  const double ddfzero = (1.0 / 3.0) * dfact * 2.0;
  const D3 sums = na + nb + 1.0e-50;
  const D3 X = d3sqrt(d3pow(K.vwn_fact / sums, K.vwn_third));
  const D3 zeta = (na - nb) / sums;
  const D3 ecpara = ap * vwn_ec3(X, bp, cp, x0p);
  const D3 ecferr = af * vwn_ec3(X, bf, cf, x0f);
  const D3 alphac = aa * vwn_ec3(X, ba, ca, x0a);
  const D3 betac = (ddfzero / alphac) * (ecferr - ecpara) - 1.0;
  const D3 fz = ffact * (d3pow(1.0 + zeta, 4.0 / 3.0) + d3pow(1.0 - zeta, 4.0 / 3.0) - 2.0);
  const D3 z2 = zeta * zeta;
  const D3 deltec = alphac * (fz / ddfzero) * (1.0 + betac * (z2 * z2));
  return (ecpara + deltec) * sums;
}

// PW92 G(rs) for the three parameter sets (1 ECU, 2 ECP, 3 -alpha_c),
// pw_ldac_module.f90:171-192 with set_param :591-651
__device__ __forceinline__ D3 pw92_g3(D3 rs, int what) {
  double a, a1, b1, b2, b3, b4;
  if (what == 1) { a = 0.031091; a1 = 0.21370; b1 = 7.5957; b2 = 3.5876; b3 = 1.6382; b4 = 0.49294; }
  else if (what == 2) { a = 0.015545; a1 = 0.20548; b1 = 14.1189; b2 = 6.1977; b3 = 3.3662; b4 = 0.62517; }
  else { a = 0.016887; a1 = 0.11125; b1 = 10.357; b2 = 3.6231; b3 = 0.88026; b4 = 0.49671; }
  const D3 rs12 = d3pow(rs, 0.5);
  const D3 Q0 = -2.0 * a * (1.0 + a1 * rs);
  const D3 Q1 = 2.0 * a * (b1 * rs12 + b2 * rs + b3 * (rs * rs12) + b4 * (rs * rs));
  return Q0 * d3log(1.0 + 1.0 / Q1);
}

// PW92 c_lda(na, nb), pw_ldac_module.f90:127-194: n * eps_c
__device__ __forceinline__ D3 pw92_c_lda(const XcConst& K, D3 na, D3 nb) {
  const double deps = 1.0e-30;
  const double cf = K.pw_cf;
  const double cfzz = 2.0 * (4.0 / 3.0) * (1.0 / 3.0) * cf;
  D3 nn = na + nb;
  if (nn.v < deps) nn = d3c(deps);  // frozen: no derivative (the reference fixes it)
  const D3 rs = K.pw_crs / d3pow(nn, 1.0 / 3.0);
  const D3 ecu = pw92_g3(rs, 1), ecp = pw92_g3(rs, 2), malf = pw92_g3(rs, 3);
  const D3 z = (na - nb) / nn;
  const D3 z2 = z * z;
  const D3 z4 = z2 * z2;
  const D3 f = cf * (d3pow(1.0 + z + deps, 4.0 / 3.0) + d3pow(1.0 - z + deps, 4.0 / 3.0) - 2.0);
  return nn * (ecu + (ecp - ecu) * f * z4 - malf * f * (1.0 - z4) / cfzz);
}

// PBE correlation H(na, nb, g2), pbe_ggcxc_module.f90:96-145: n * H;
// g2 = |grad n|^2 of the total density
__device__ __forceinline__ D3 pbe_c_gga(const XcConst& K, D3 na, D3 nb, D3 g2) {
  const double beta = K.pbe_beta, gam = 0.03109069086965489503494086371, deps = 1.0e-30;
  const D3 n = na + nb;
  if (n.v <= 0.0) return d3c(0.0);
  const D3 eldac = pw92_c_lda(K, na, nb) / n;
  D3 za = na / n, zb = nb / n;
  if (za.v < deps) za = d3c(deps);
  if (zb.v < deps) zb = d3c(deps);
  const D3 fi = (d3pow(za, 2.0 / 3.0) + d3pow(zb, 2.0 / 3.0)) * K.pbe_two13i;
  const D3 fi2 = fi * fi;
  const D3 fi3 = fi2 * fi;
  const D3 A = (beta / gam) / (d3exp(-eldac / (gam * fi3)) - 1.0 + deps);
  const D3 t2 = g2 / (fi2 * d3pow(n, 7.0 / 3.0) + deps) * K.pbe_ct;
  const D3 x = A * t2;
  const D3 rat = (1.0 + x) / (1.0 + x + x * x);
  return n * (gam * fi3 * d3log(1.0 + (beta / gam) * t2 * rat));
}

// PW91 correlation H0 + H1 (pbe_or_pw91 with H_pw91, H0_drv, H1_drv, F_drv,
// S_drv, Cc_drv, Hln_drv, A_drv; modules/gga_response_module.f90:278-918,
// parameters :150-156): n * H(na, nb, g2) with ec = n eps_c of the LDA
// correlation that precedes it.  The floors of n (1e-20) replace values only:
// the derivative formulas keep treating n as the variable, as the reference's do.
__device__ __forceinline__ D3 pw91_c_gga(const XcConst& K, D3 na, D3 nb, D3 g2, D3 ec) {
  const double eps = 1.0e-20, pi = 3.14159265358979324;
  const double alpha = 0.09, nu = 15.755920349483144658863574030524, cc0 = 0.004235, cx = -0.001667;
  const double beta = nu * cc0, gam = beta * beta / (2.0 * alpha), bdg = beta / gam;
  D3 nn = na + nb;
  if (fabs(nn.v) < eps) nn.v = eps;
  const D3 rs = 1.91916 / d3pow((3.0 * pi * pi) * nn, 1.0 / 3.0);
  // phi = ((1+z)^(2/3) + (1-z)^(2/3)) / 2; its derivatives in na, nb as the
  // reference writes them (with eps under the cube roots)
  const double z = (na.v - nb.v) / nn.v;
  const double phv = 0.5 * (pow(1.0 + z, 2.0 / 3.0) + pow(1.0 - z, 2.0 / 3.0));
  const double pf = (1.0 / 3.0) * pow(2.0, 2.0 / 3.0) / pow(nn.v, 5.0 / 3.0);
  const double pa = pf * (nb.v / pow(na.v + eps, 1.0 / 3.0) - pow(nb.v, 2.0 / 3.0));
  const double pb = pf * (na.v / pow(nb.v + eps, 1.0 / 3.0) - pow(na.v, 2.0 / 3.0));
  const D3 p = D3{phv, {pa * na.d[0] + pb * nb.d[0], pa * na.d[1] + pb * nb.d[1], pa * na.d[2] + pb * nb.d[2]}};
  const D3 pn = p * d3pow(nn, 7.0 / 6.0);
  const D3 t = K.pbe_ct * g2 / (pn * pn);  // t^2
  const D3 e = ec / nn;                     // eps_c of the LDA
  const D3 p2 = p * p, p3 = p2 * p;
  // H0 = gamma phi^3 ln(1 + g), A = (beta/gamma) / (exp(-e / (gamma phi^3)) - 1)
  const D3 xe = -e / (gam * p3);
  D3 A = bdg / ((d3exp(xe) - 1.0) + eps);
  if (xe.v > 300.0) A.d[0] = A.d[1] = A.d[2] = 0.0;
  const D3 at = A * t;
  const D3 at1 = 1.0 + at;
  const D3 at2 = at1 + at * at;
  const D3 g = (bdg * t) * (at1 / at2);
  const D3 h0 = gam * p3 * d3log(1.0 + g);
  // H1 = nu (Cc(rs) - Cc0 - 3 Cx / 7) phi^3 t^2 exp(-100 phi^4 (ks/kF)^2 t^2)
  const D3 rs2 = rs * rs;
  const D3 fup = 2.568 + 23.266 * rs + 0.007389 * rs2;
  const D3 fdn = 1.0 + 8.723 * rs + 0.472 * rs2 + 0.073890 * (rs2 * rs);
  const D3 cc = fup / fdn / 1000.0 - cx;
  const D3 F = nu * (cc - cc0 - (3.0 / 7.0) * cx) * p3 * t;
  const double ksf = 4.0 / (1.91916 * pi);
  const D3 S = d3exp(-100.0 * (p3 * p) * t * ksf * rs);
  return nn * (h0 + F * S);
}

// LYP correlation in the form of lyp_corr (modules/lyp.f90, parameter set 1)
// for spin densities ra, rb; it is linear in the gradient invariants, so the
// coefficients c[0..2] of gaa, gbb, gab are returned beside the value:
// F = F0(ra, rb) + c[0] gaa + c[1] gbb + c[2] gab, with derivatives in ra, rb.
__device__ __forceinline__ D3 lyp_corr(const XcConst& K, D3 ra, D3 rb, double gaa, double gbb, double gab,
                                       double (&c)[3]) {
  const double a = 0.04918, b = 0.13200, cp = 0.25330, d = 0.34900, e = 2.87123400018819, tol = 1.0e-30;
  const D3 rsum = ra + rb;
  const bool live = rsum.v > tol;
  D3 qz = d3c(0.0), qw = d3c(0.0), qd = d3c(0.0);
  if (live) {
    const D3 r13 = d3pow(rsum, 1.0 / 3.0);
    qz = r13 / (d + r13);
    qw = d3exp(-cp / r13) * qz * d3pow(rsum, -11.0 / 3.0);
    qd = (cp + d * qz) / r13;
  }
  const D3 f1 = (a * b) * qw;
  const D3 f2 = f1 * ra * rb;
  const D3 lda1 = live ? 4.0 * a * ra * rb * qz / rsum : d3c(0.0);
  const D3 lda2 = f2 * K.lyp_2113 * e * (d3pow(ra, 8.0 / 3.0) + d3pow(rb, 8.0 / 3.0));
  const D3 base = 1.0 / 9.0 - (1.0 / 3.0) * qd;
  const D3 caa = (live ? f2 * (base - (1.0 / 9.0) * (qd - 11.0) * ra / rsum) : f2 * base) - f1 * (rb * rb);
  const D3 cbb = (live ? f2 * (base - (1.0 / 9.0) * (qd - 11.0) * rb / rsum) : f2 * base) - f1 * (ra * ra);
  const D3 cab = f2 * (47.0 / 9.0 - (7.0 / 9.0) * qd) - f1 * (4.0 / 3.0) * (rsum * rsum);
  c[0] = -caa.v;
  c[1] = -cbb.v;
  c[2] = -cab.v;
  return -lda1 - lda2 - caa * gaa - cbb * gbb - cab * gab;
}

// LB94 potential correction of one spin density (baerends94_calc,
// modules/baerends_module.f90:91-134): -beta r^(1/3) x^2 / (1 + 3 beta x
// asinh x), x = c |grad r| / (r + 1e-50)^(4/3), asinh as log(x + sqrt(x^2 + 1));
// beta is the reference's single-precision 0.05.  Closed shell: r = n,
// c = 2^(1/3) and the result divided by 2^(1/3); open shell: c = 1.
__device__ __forceinline__ double lb94_dv(double r, double gam, double c) {
  const double beta = (double)0.05f;
  const double x = c * sqrt(gam) / pow(r + 1.0e-50, 4.0 / 3.0);
  const double den = 1.0 + 3.0 * beta * x * log(x + sqrt(x * x + 1.0));
  return beta * pow(r, 1.0 / 3.0) * x * x / den;
}

// HCTH power series g(s2) = sum_n c_n u^n, u = s2 / (1 + s2), and dg/ds2
// (hcth.f90 g, in hcth_x_calc and hcth_c_calc).
__device__ __forceinline__ void hcth_g(const double (&c)[5], double s2, double& g0, double& g1) {
  const double u = s2 / (1.0 + s2);
  const double du = 1.0 / ((1.0 + s2) * (1.0 + s2));
  double a = 0.0, b = 0.0;
#pragma unroll
  for (int n = 4; n >= 1; --n) {
    a = c[n] + u * a;
    b = n * c[n] + u * b;
  }
  g0 = c[0] + u * a;
  g1 = b * du;
}

// HCTH at one point of spin densities ra, rb and gamma_aa, gamma_bb (it has no
// gamma_ab dependence): hcth_x_calc and hcth_c_calc (hcth.f90).  Adds f,
// fr[0..1], fg[0..1].
__device__ __forceinline__ void hcth_point(const XcConst& K, double ra, double rb, double gaa, double gbb, double& f,
                                           double* fr, double* fg) {
  const double deps = 1.0e-15;
  // exchange, per spin: e_x,s g_x(0.004 gamma_ss / rho_s^(8/3))
  const double rs[2] = {ra, rb}, gs[2] = {gaa, gbb};
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double r = rs[s];
    if (r < deps) continue;
    const double c = cbrt(r);
    const double ex = K.hcth_xa * r * c;
    const double dex = K.hcth_xa * c * (4.0 / 3.0);
    const double r83 = r * r * c * c;
    const double s2 = 0.004 * gs[s] / r83;
    double u, du;
    hcth_g(K.hcth_x, s2, u, du);
    f += ex * u;
    fr[s] += ex * du * (-(8.0 / 3.0) * s2 / r) + dex * u;
    fg[s] += ex * du * (0.004 / r83);
  }
  // correlation: e_aa g_aa(0.2 s_aa^2) + e_bb g_aa(0.2 s_bb^2) + e_ab g_ab(0.006 s_avg^2),
  // e_ss = PW92 of the fully polarised density rho_s, e_ab = PW92(ra, rb) - e_aa - e_bb
  if (ra + rb < deps) return;
  const D3 na = d3v(0, ra), nb = d3v(1, rb);
  const D3 eaa = pw92_c_lda(K, na, d3c(0.0));
  const D3 ebb = pw92_c_lda(K, nb, d3c(0.0));
  const D3 eab = pw92_c_lda(K, na, nb) - eaa - ebb;
  const double ma = fmax(ra, deps), mb = fmax(rb, deps);
  const double ca = cbrt(ma), cb = cbrt(mb);
  const double ia = 1.0 / (ma * ma * ca * ca), ib = 1.0 / (mb * mb * cb * cb);  // rho^(-8/3)
  const double saa = gaa * ia, sbb = gbb * ib, sab = 0.5 * (saa + sbb);
  const double daa = -(8.0 / 3.0) * saa / ma, dbb = -(8.0 / 3.0) * sbb / mb;
  double uaa, duaa, ubb, dubb, uab, duab;
  hcth_g(K.hcth_caa, 0.2 * saa, uaa, duaa);
  hcth_g(K.hcth_caa, 0.2 * sbb, ubb, dubb);
  hcth_g(K.hcth_cab, 0.006 * sab, uab, duab);
  f += eaa.v * uaa + ebb.v * ubb + eab.v * uab;
  fr[0] += eaa.d[0] * uaa + eaa.v * duaa * (0.2 * daa) + eab.d[0] * uab + eab.v * duab * (0.006 * 0.5 * daa);
  fr[1] += ebb.d[1] * ubb + ebb.v * dubb * (0.2 * dbb) + eab.d[1] * uab + eab.v * duab * (0.006 * 0.5 * dbb);
  fg[0] += eaa.v * duaa * (0.2 * ia) + eab.v * duab * (0.006 * 0.5 * ia);
  fg[1] += ebb.v * dubb * (0.2 * ib) + eab.v * duab * (0.006 * 0.5 * ib);
}

// Perdew 86 gradient correlation with its first derivatives (perdew_calc,
// modules/becke_perdew_module.f90:125-260; constants :83-118).  ispin = 1:
// rho[0], gam[0]; ispin = 2: rho[0..1], gam = (aa, bb, ab), the correlation
// of the total gradient scaled by the spin factor d(zeta).  Adds f, fr, fg.
__device__ __forceinline__ void perdew86(int ispin, const double* rho, const double* gam, double& f, double* fr,
                                         double* fg) {
  const double deps = 1.0e-30, third = 1.0 / 3.0;
  const double alpha = 0.023266, beta = 7.389e-6, gammas = 8.723, delta = 0.472;
  const double cfac = 0.001667, ocfac = 0.002568, rs_fac = 0.62035049089940001667;
  const double fi_fac = 1.745 * 0.11 * (cfac + ocfac);
  const double e4_beta = beta * 1.0e4, two_oth = 1.25992104989487316476;
  double sums, xi_u = 0, xi_d = 0, dm = 1.0, ddm_xi = 0;
  if (ispin == 1) {
    sums = rho[0] + deps;
  } else {
    sums = rho[0] + rho[1] + deps;
    const double xi = (rho[0] - rho[1]) / sums;
    xi_u = (1.0 - xi) / sums;
    xi_d = -(1.0 + xi) / sums;
    const double up = (1.0 + xi) / 2.0, dn = (1.0 - xi) / 2.0;
    dm = (1.0 / two_oth) / sqrt(pow(up, 5.0 / 3.0) + pow(dn, 5.0 / 3.0));
    ddm_xi = (5.0 / 12.0) * dm * dm * dm * two_oth * two_oth * (pow(dn, 2.0 / 3.0) - pow(up, 2.0 / 3.0));
  }
  const double rothrd = cbrt(sums), rof4th = sums * rothrd;
  const double rs = rs_fac / rothrd, rs2 = rs * rs, rs3 = rs2 * rs;
  const double gr2 = ispin == 1 ? gam[0] : gam[0] + gam[1] + 2.0 * gam[2];
  const double gr = sqrt(gr2);
  const double cden = 1.0 + gammas * rs + delta * rs2 + e4_beta * rs3;
  const double ovcf = ocfac + alpha * rs + beta * rs2;
  const double c_rho = cfac + ovcf / cden;
  const double r76 = sums * sqrt(rothrd);  // sums^(7/6)
  const double fi_g = fi_fac / (c_rho * r76);
  const double exp_fi = exp(-fi_g * gr);
  const double dP_g = (exp_fi * c_rho / rof4th) * (1.0 - fi_g * gr / 2.0);
  const double t1 = (alpha + 2.0 * beta * rs) / cden;
  const double t2 = (gammas + 2.0 * delta * rs + 3.0 * e4_beta * rs2) * ovcf / (cden * cden);
  const double dC = -third * rs / sums * (t1 - t2);
  const double cr = c_rho * r76;
  const double dfi_rho = -(fi_fac / (cr * cr)) * sqrt(rothrd) * (dC * sums + (7.0 / 6.0) * c_rho) * gr;
  const double P = c_rho / rof4th * exp_fi * gr2;
  const double dP_rho = (exp_fi / rof4th) * (dC - (4.0 / 3.0) * c_rho / sums - c_rho * dfi_rho) * gr2;
  if (ispin == 1) {
    f += P;
    fr[0] += dP_rho;
    fg[0] += dP_g;
  } else {
    f += P * dm;
    fr[0] += dP_rho * dm + ddm_xi * xi_u * P;
    fr[1] += dP_rho * dm + ddm_xi * xi_d * P;
    fg[0] += dP_g * dm;
    fg[1] += dP_g * dm;
    fg[2] += 2.0 * dP_g * dm;
  }
}

// "BP": Slater + VWN5 + Becke 88 exchange + Perdew 86 correlation
// (modules/xc_cntrl.f90:508-520); n = total density, g = |grad n|^2.
__device__ __forceinline__ void xc_bp86(const XcConst& K, double n, double g, double& f, double& fr, double& fg) {
  xc_vwn(K, n, f, fr);  // Slater + VWN5
  fg = 0.0;
  pbe_x(K, n, g, f, fr, fg);  // K.xg == XG_B88
  double pf = 0.0, pr = 0.0, pg = 0.0;
  perdew86(1, &n, &g, pf, &pr, &pg);
  f += K.fc_g * pf;
  fr += K.fc_g * pr;
  fg += K.fc_g * pg;
}

// The PW91 correlation of the older pw91c_calc (perdew_wang_module.f90:112-490,
// not revised) with its closed-form derivatives as written there: n floored at
// 1e-50, 1 +- zeta at 1e-25, exp(.) - 1 of A at 1e-50, 1e-50 added under
// dt/dgamma, and (open shell) dH1/drs without the g^3 of H1.  ec, ecr: the LDA
// correlation per volume and its density derivatives.  f = n H; fr[s], fg[k].
__device__ __forceinline__ void pw91c_old(bool open, const double* rho, const double* gam, double ec,
                                          const double* ecr, double& f, double* fr, double* fg) {
  const double pi = 3.141592653589793240, deps = 1.0e-50;
  const double Cc0 = 0.004235, Cx = -0.001667, al = 0.09, Cx37 = Cx * 3.0 / 7.0;
  const double a_rg = 23.266, b_rg = 7.389e-3, c_rg = 8.723, d_rg = 0.472, e_rg = 2.568;
  const double cr3pi2 = cbrt(3.0 * pi * pi);
  const double rs_fact = cbrt(3.0 / (4.0 * pi)), h1_fact = (16.0 / pi) * cr3pi2;
  const double bpw = h1_fact * Cc0, h0_fact = bpw * bpw / (2.0 * al), apf = 2.0 * al / bpw;
  const double t_fact = 1.0 / (2.0 * sqrt(cbrt(192.0 / pi)));
  const double e_fact = 100.0 * 4.0 / (pi * cr3pi2);
  double n = open ? rho[0] + rho[1] : rho[0];
  if (n < deps) n = deps;
  const double eps = ec / n;
  const double rt = cbrt(n), rs = rs_fact / rt, rs2 = rs * rs;
  double pa = 1.0, pb = 1.0;
  if (open) {
    const double zeta = (rho[0] - rho[1]) / n;
    pa = fmax(1.0 + zeta, 1.0e-25);
    pb = fmax(1.0 - zeta, 1.0e-25);
  }
  const double g = open ? 0.5 * (pow(pa, 2.0 / 3.0) + pow(pb, 2.0 / 3.0)) : 1.0;
  const double g2 = g * g, g3 = g2 * g, g4 = g2 * g2;
  const double gr = sqrt(open ? gam[0] + gam[1] + 2.0 * gam[2] : gam[0]);
  const double srt = sqrt(rt);
  const double t = t_fact * gr / (srt * n) / g, t2 = t * t;
  const double t_g = 0.5 * t_fact / (srt * n * gr + deps) / g;
  const double t_n = -(7.0 / 6.0) * t / n, t_gi = -t / g;
  const double ex0 = -2.0 * al * eps / (bpw * bpw) / g3;
  const double V = exp(ex0);
  const double Aden = fmax(V - 1.0, deps);
  const double A = apf / Aden, At2 = A * t2, OA = 1.0 + At2;
  const double den = (1.0 + (apf + A) * t2 * OA) * (OA + At2 * At2);
  const double h0 = g3 * h0_fact * log(1.0 + apf * (t2 + At2 * t2) / (OA + At2 * At2));
  const double F0_t = g3 * n * 2.0 * bpw * t * (OA + At2) / den;
  const double h0_a = -g3 * bpw * t2 * t2 * t2 * A * (2.0 + At2) / den;
  const double ex1 = -g4 * e_fact * t2 / rt, E1 = exp(ex1);
  const double rn = e_rg + a_rg * rs + b_rg * rs2, rd = 1.0 + c_rg * rs + d_rg * rs2 + 10.0 * b_rg * rs2 * rs;
  const double K1 = h1_fact * (1.0e-3 * rn / rd - Cx - Cc0 - Cx37);
  const double h1 = g3 * K1 * t2 * E1;
  const double h1_t = g3 * K1 * E1 * 2.0 * t * (1.0 + ex1);
  const double rn1 = a_rg + 2.0 * b_rg * rs, rd1 = c_rg + 2.0 * d_rg * rs + 30.0 * b_rg * rs2;
  const double h_rs = h1_fact * t2 * E1 * 1.0e-3 * (rn1 * rd - rd1 * rn) / (rd * rd);
  const double rs_n = -rs / (3.0 * n);
  const double h1_dn = g4 * h1 * t2 * e_fact / (3.0 * n * rt);
  const double Fg = F0_t * t_g + n * h1_t * t_g;
  const double vA = V / (Aden * Aden);
  f = (h0 + h1) * n;
  if (!open) {
    const double A_n = (apf * apf / bpw) * vA * (ecr[0] - eps) / n;
    fr[0] = h0 + n * h0_a * A_n + F0_t * t_n + h1 + n * (h_rs * rs_n + h1_t * t_n + h1_dn);
    fg[0] = Fg;
    return;
  }
  const double A_gi = 3.0 * (apf * vA) * ex0 * g3 / g4;
  const double dg = (1.0 / 3.0) * (1.0 / cbrt(pa) - 1.0 / cbrt(pb));
  const double h0_t = F0_t / n, h0_gi = 3.0 * g2 / g3 * h0;
  const double h1_gi = 3.0 * g2 / g3 * h1 + h1 * (4.0 * g3 / g4) * ex1;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double zs = s == 0 ? pb / n : -pa / n;
    const double A_ns = (apf * apf / (bpw * g3)) * vA * (ecr[s] - eps) / n + A_gi * dg * zs;
    const double h0_ns = h0_gi * dg * zs + h0_a * A_ns + h0_t * (t_n + t_gi * dg * zs);
    const double h1_ns = h1_t * t_gi * dg * zs + h1_t * t_n + h1_gi * dg * zs + h_rs * rs_n + h1_dn;
    fr[s] = h0 + n * h0_ns + h1 + n * h1_ns;
  }
  fg[0] = fg[1] = Fg;
  fg[2] = 2.0 * Fg;
}

// "RPW91"'s correction (xc_rperdewwang91c, xc_func.f90:436-446): the H of
// pw91c_calc times phi_c(b) = (1 + a1 b^2 + a2 b^4) / (1 + b1 b^2 + b2 b^4),
// b = (3 pi^2 n)^(1/3) / c, n floored at 1e-50; rpw91c_calc scales F first and
// then adds the scaled F times dphi_c/dn to dF/drho (relxc.f90:162-218).
__device__ __forceinline__ void rpw91c_add(const XcConst& K, bool open, const double* rho, const double* gam,
                                           double ec, const double* ecr, double& f, double* fr, double* fg) {
  double h, hr[2], hg[3];
  pw91c_old(open, rho, gam, ec, ecr, h, hr, hg);
  const double a1 = 1.9407, a2 = 0.14435, b1 = 0.28412, b2 = 0.004723;
  const double n = fmax(open ? rho[0] + rho[1] : rho[0], 1.0e-50);
  const double b = cbrt(K.rel_3pi2 * n) / K.rel_c, bb = b * b;
  const double num = 1.0 + a1 * bb + a2 * bb * bb, den = 1.0 + b1 * bb + b2 * bb * bb;
  const double phi = num / den;
  const double dphi = (den * (2.0 * a1 * b + 4.0 * a2 * bb * b) - num * (2.0 * b1 * b + 4.0 * b2 * bb * b)) * b /
                      (3.0 * n * den * den);
  const double hs = h * phi;
  f += hs;
  const int ns = open ? 2 : 1, ng = open ? 3 : 1;
  for (int s = 0; s < ns; ++s) fr[s] += hr[s] * phi + hs * dphi;
  for (int k = 0; k < ng; ++k) fg[k] += hg[k] * phi;
}

// "PW91", "BPW91" (PW92 + PW91 correlation), "BLYP" (LYP) and "B88" (no
// correlation), closed shell, through the dual numbers in (n, g) or, for
// LYP, in (rho_a, rho_b).
__device__ __forceinline__ void xc_gga_d3(const XcConst& K, double n, double g, double& f, double& fr, double& fg) {
  f = 0.0;
  fr = 0.0;
  fg = 0.0;
  slater(K, n, f, fr);
  pbe_x(K, n, g, f, fr, fg);
  // LDA correlation at na = nb = n/2: PW92 (pw_ldac), VWN5 (B3LYP) or none
  const D3 nv = d3v(0, n);
  const D3 na = 0.5 * nv, nb = 0.5 * nv;
  D3 ec = d3c(0.0);
  if (K.lc == LC_PW92) ec = pw92_c_lda(K, na, nb);
  else if (K.lc == LC_VWN) ec = vwn_c_lda(K, na, nb);
  f += K.fc_lda * ec.v;
  fr += K.fc_lda * ec.d[0];
  if (K.cg == CG_PW91) {
    // gga_correlation (gga_response_module.f90:170-275): na = nb = n/2, the
    // (unscaled) LDA energy of pw_ldac
    const D3 c = pw91_c_gga(K, na, nb, d3v(1, g), ec);
    f += K.fc_g * c.v;
    fr += K.fc_g * c.d[0];
    fg += K.fc_g * c.d[1];
    if (K.rpw91c) {
      const double ecr = ec.d[0];
      rpw91c_add(K, false, &n, &g, ec.v, &ecr, f, &fr, &fg);
    }
  } else if (K.cg == CG_LYP) {
    // lyp_C (lyp.f90): ra = rb = n/2, gaa = gbb = gab = g/4; dF/dn is dF/dra
    // and dF/dg is the coefficient of gaa alone, as the reference returns them
    const double q = 0.25 * g;
    double c3[3];
    const D3 F = lyp_corr(K, d3v(0, 0.5 * n), d3v(1, 0.5 * n), q, q, q, c3);
    f += K.fc_g * F.v;
    fr += K.fc_g * F.d[0];
    fg += K.fc_g * c3[0];
  }
  if (K.lb94) {
    const double two13 = K.lb94_two13;
    fr -= lb94_dv(n, g, two13) / two13;
  }
}

// HCTH, closed shell (pg_hcth, hcth.f90): ra = rb = n/2, gaa = gbb = g/4,
// df/dn = (df/dra + df/drb)/2, df/dg = (df/dgaa + df/dgbb)/4.
__device__ __forceinline__ void xc_hcth(const XcConst& K, double n, double g, double& f, double& fr, double& fg) {
  double r2[2] = {0.0, 0.0}, g2[2] = {0.0, 0.0};
  f = 0.0;
  hcth_point(K, 0.5 * n, 0.5 * n, 0.25 * g, 0.25 * g, f, r2, g2);
  fr = 0.5 * (r2[0] + r2[1]);
  fg = 0.25 * (g2[0] + g2[1]);
}

// The closed-shell GGA keyword of K.
__device__ __forceinline__ void xc_gga(const XcConst& K, double n, double g, double& f, double& fr, double& fg) {
  if (K.hcth) xc_hcth(K, n, g, f, fr, fg);
  else if (K.cg == CG_PBE && K.lc == LC_PW92) xc_pbe(K, n, g, f, fr, fg);
  else if (K.cg == CG_P86) xc_bp86(K, n, g, f, fr, fg);
  else xc_gga_d3(K, n, g, f, fr, fg);
}

// GGA terms of the open-shell functional: exchange enhancement and gradient
// correlation; ec = the LDA correlation already added (n eps_c, D3 in na, nb).
__device__ __forceinline__ void xc_open_gga(const XcConst& K, const double (&rho)[2], const double (&gam)[3], D3 na,
                                            D3 nb, D3 ec, double& f, double (&fr)[2], double (&fg)[3]) {
  // exchange enhancement, spin-scaled: e(2 rho_s, 4 gamma_ss) / 2
  for (int s = 0; s < 2; ++s) {
    double F = 0.0, Fn = 0.0, Fg = 0.0;
    pbe_x(K, 2.0 * rho[s], 4.0 * gam[s], F, Fn, Fg);
    f += 0.5 * F;
    fr[s] += Fn;
    fg[s] += 2.0 * Fg;
  }
  if (K.lb94) {
    fr[0] -= lb94_dv(rho[0], gam[0], 1.0);
    fr[1] -= lb94_dv(rho[1], gam[1], 1.0);
  }
  if (K.cg == CG_NONE) return;
  const double a = K.fc_g;
  if (K.cg == CG_P86) {
    double pf = 0.0, pr[2] = {0.0, 0.0}, pg[3] = {0.0, 0.0, 0.0};
    perdew86(2, rho, gam, pf, pr, pg);
    f += a * pf;
    fr[0] += a * pr[0];
    fr[1] += a * pr[1];
    fg[0] += a * pg[0];
    fg[1] += a * pg[1];
    fg[2] += a * pg[2];
    return;
  }
  if (K.cg == CG_LYP) {
    double c3[3];
    const D3 F = lyp_corr(K, na, nb, gam[0], gam[1], gam[2], c3);
    f += a * F.v;
    fr[0] += a * F.d[0];
    fr[1] += a * F.d[1];
    fg[0] += a * c3[0];
    fg[1] += a * c3[1];
    fg[2] += a * c3[2];
    return;
  }
  // PBE or PW91 correlation H of the total gradient |grad rho_a + grad rho_b|^2
  D3 g2 = d3v(2, gam[0] + gam[1] + 2.0 * gam[2]);
  D3 c;
  if (K.cg == CG_PW91) {
    if (g2.v < 1.0e-20) g2.v = 1.0e-20;  // gga_correlation's floor of gm
    c = pw91_c_gga(K, na, nb, g2, ec);
  } else {
    c = pbe_c_gga(K, na, nb, g2);
  }
  f += a * c.v;
  fr[0] += a * c.d[0];
  fr[1] += a * c.d[1];
  fg[0] += a * c.d[2];
  fg[1] += a * c.d[2];
  fg[2] += a * 2.0 * c.d[2];
  if (K.rpw91c) {
    const double ecr[2] = {ec.d[0], ec.d[1]};
    rpw91c_add(K, true, rho, gam, ec.v, ecr, f, fr, fg);
  }
}

// Open-shell functional at one point: rho[2] = (rho_a, rho_b), gam[3] =
// (gamma_aa, gamma_bb, gamma_ab); f, fr[2] = df/drho_s, fg[3] = df/dgamma_*.
// xc_functionals composition (xc_func.f90:187-305), as for ispin = 1.
template <bool GGA>
__device__ __forceinline__ void xc_open(const XcConst& K, const double (&rho)[2], const double (&gam)[3], double& f,
                                        double (&fr)[2], double (&fg)[3]) {
  f = 0.0;
  fr[0] = fr[1] = 0.0;
  fg[0] = fg[1] = fg[2] = 0.0;
  if (GGA && K.hcth) {
    hcth_point(K, rho[0], rho[1], gam[0], gam[1], f, fr, fg);
    return;
  }
  // Slater, spin-scaled
  for (int s = 0; s < 2; ++s) {
    double F = 0.0, Fn = 0.0;
    slater(K, 2.0 * rho[s], F, Fn);
    f += F / 2.0;
    fr[s] += Fn;
  }
  const D3 na = d3v(0, rho[0]), nb = d3v(1, rho[1]);
  // LDA correlation: VWN5 ("VWN", "BP"), PW92, or none ("XALPHA", "B88", "BLYP")
  D3 ec = d3c(0.0);
  if (K.lc == LC_VWN) ec = vwn_c_lda(K, na, nb);
  else if (K.lc == LC_PW92) ec = pw92_c_lda(K, na, nb);
  f += K.fc_lda * ec.v;
  fr[0] += K.fc_lda * ec.d[0];
  fr[1] += K.fc_lda * ec.d[1];
  if (K.rvwn == 1) {  // rel_vwn_calc: a function of the total density
    double er, der;
    rel_vwn(K, rho[0] + rho[1], er, der);
    f += er;
    fr[0] += der;
    fr[1] += der;
  } else if (K.rvwn == 2) {  // correlation_lda: VWN5 (phic0(beta(n)) - 1), n = rho_a + rho_b
    double p, dp;
    engel_phic0(K, rho[0] + rho[1], p, dp);
    f += ec.v * (p - 1.0);
    fr[0] += ec.d[0] * (p - 1.0) + ec.v * dp;
    fr[1] += ec.d[1] * (p - 1.0) + ec.v * dp;
  }
  if constexpr (GGA) xc_open_gga(K, rho, gam, na, nb, ec, f, fr, fg);
}

}  // namespace pgxc
