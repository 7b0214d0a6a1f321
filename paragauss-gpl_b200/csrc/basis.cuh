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

// Y[l*l + m] and dY[c][l*l + m], c = x, y, z, for l <= L, in real type R.
template <int L, typename R>
__device__ __forceinline__ void solid_harmonics(R x, R y, R z, R* Y, R (*dY)[16]) {
  const R r2 = x * x + y * y + z * z;
  Y[0] = R(1);
  dY[0][0] = dY[1][0] = dY[2][0] = R(0);
  if (L == 0) return;
  Y[1] = z; Y[2] = x; Y[3] = y;
  dY[0][1] = 0; dY[1][1] = 0; dY[2][1] = 1;
  dY[0][2] = 1; dY[1][2] = 0; dY[2][2] = 0;
  dY[0][3] = 0; dY[1][3] = 1; dY[2][3] = 0;
#pragma unroll
  for (int l = 2; l <= L; ++l) {
    const int o = l * l, o1 = (l - 1) * (l - 1), o2 = (l - 2) * (l - 2);
    const R lr = R(l), l1r = R(l - 1), ll1r = R(2 * l - 1);
    const R dr2[3] = {R(2) * x, R(2) * y, R(2) * z};
    // m index 0
    {
      const R p1 = Y[o1], p2 = Y[o2];
      Y[o] = (ll1r * z * p1 - l1r * r2 * p2) / lr;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        dY[c][o] = (ll1r * ((c == 2 ? p1 : R(0)) + z * dY[c][o1]) - l1r * (dr2[c] * p2 + r2 * dY[c][o2])) / lr;
    }
#pragma unroll
    for (int im = 1; im <= l - 2; ++im) {
      const R sim = (R)(im * im);
      const R rlm = R(1) / sqrt(lr * lr - sim);
      const R rl1m = sqrt(l1r * l1r - sim);
      const R a = ll1r * z * rlm;
      const R b = rl1m * r2 * rlm;
#pragma unroll
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const R p1 = Y[o1 + mm], p2 = Y[o2 + mm];
        Y[o + mm] = a * p1 - b * p2;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : R(0)) + a * dY[c][o1 + mm] - rl1m * dr2[c] * rlm * p2 -
                          b * dY[c][o2 + mm];
      }
    }
    {
      const int im = l - 1;
      const R rlm = R(1) / sqrt(lr * lr - (R)(im * im));
      const R a = ll1r * z * rlm;
#pragma unroll
      for (int mm = 2 * im - 1; mm <= 2 * im; ++mm) {
        const R p1 = Y[o1 + mm];
        Y[o + mm] = a * p1;
#pragma unroll
        for (int c = 0; c < 3; ++c) dY[c][o + mm] = (c == 2 ? ll1r * rlm * p1 : R(0)) + a * dY[c][o1 + mm];
      }
    }
    {
      const R rll = sqrt(ll1r / (R(2) * lr));
      const R q2 = Y[o1 + 2 * l - 3], q1 = Y[o1 + 2 * l - 2];
      Y[o + 2 * l - 1] = (x * q2 - y * q1) * rll;
      Y[o + 2 * l] = (y * q2 + x * q1) * rll;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const R g2 = dY[c][o1 + 2 * l - 3], g1 = dY[c][o1 + 2 * l - 2];
        const R dx = R(c == 0), dy = R(c == 1);
        dY[c][o + 2 * l - 1] = (dx * q2 + x * g2 - dy * q1 - y * g1) * rll;
        dY[c][o + 2 * l] = (dy * q2 + y * g2 + dx * q1 + x * g1) * rll;
      }
    }
  }
}

// One normalised primitive norm*exp(-alpha r^2), zero where alpha r^2 >= 50
// (radial0/radial1, modules/orbital_module.f90:1823-1854).  In FP32 the
// exponent alpha*r^2 (up to 50) would carry an absolute rounding error of
// up to 50 * 2^-24 into exp; it is therefore formed in FP64 from the FP64 r^2
// and split as 2^-t = 2^-k * 2^-f (k integer, |f| <= 1/2) before exp2f.
__device__ __forceinline__ double prim_value(double alpha, double norm, double r2, double) {
  const double ar2 = alpha * r2;
  return ar2 < 50.0 ? norm * exp(-ar2) : 0.0;
}
__device__ __forceinline__ float prim_value(float, float norm, float, double ar2) {
  if (!(ar2 < 50.0)) return 0.f;
  const double t = ar2 * 1.4426950408889634;  // log2(e)
  const double k = rint(t);
  return norm * ldexpf(exp2f(-(float)(t - k)), -(int)k);
}

// Evaluate one shell at one point and store its (2l+1)*nrad functions (and
// gradients when GRAD) at column p of the [function][ld] arrays.  R is the
// arithmetic type (FP64 for the drop-in path, FP32 for the mixed path), T the
// stored type.  With R = float, r2d is the FP64 r^2 used for the exponent.
// exps/norms/contr may point to shared memory (plain loads).
template <int L, bool GRAD, typename T, typename R = double>
__device__ __forceinline__ void shell_at_point(const DevShell& S, const DevSA& sa, R x, R y, R z,
                                               const double* exps, const double* norms, const double* contr,
                                               bool valid, int64_t p, int64_t ld,
                                               T* __restrict__ phi, T* __restrict__ gx, T* __restrict__ gy,
                                               T* __restrict__ gz, double r2d = 0.0) {
  constexpr int NY = (L + 1) * (L + 1);
  R Y[16];
  R dY[3][16];
  solid_harmonics<L, R>(x, y, z, Y, dY);
  const R r2 = x * x + y * y + z * z;
  // symmetry-adapted harmonics of this l
  R Ys[2 * L + 1], dYs[3][2 * L + 1];
#pragma unroll
  for (int i = 0; i < 2 * L + 1; ++i) {
    if (sa.identity) {
      Ys[i] = Y[L * L + i];
#pragma unroll
      for (int c = 0; c < 3; ++c) dYs[c][i] = dY[c][L * L + i];
    } else {
      R v = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m) {
        const R cf = (R)sa.c[L][i][m];
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
    R Rr[kRadGroup], dR[kRadGroup];
#pragma unroll
    for (int r = 0; r < kRadGroup; ++r) { Rr[r] = R(0); dR[r] = R(0); }
    if (valid) {
      for (int e = 0; e < S.nexp; ++e) {
        const double alpha_d = ex[e];
        const R alpha = (R)alpha_d;
        const R v = prim_value(alpha, (R)nr[e], r2, alpha_d * r2d);
        const R dv = (R(-2) * alpha) * v;
#pragma unroll
        for (int r = 0; r < kRadGroup; ++r) {
          const int rr = r0 + r;
          if (rr < S.nrad) {
            R cf;
            if (rr < S.nunc) cf = (e == rr) ? R(1) : R(0);
            else cf = (R)cc[e + (int64_t)S.nexp * (rr - S.nunc)];
            Rr[r] += cf * v;
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
          phi[f * ld + p] = (T)(Ys[i] * Rr[r]);
          if (GRAD) {
            const R h = Ys[i] * dR[r];
            gx[f * ld + p] = (T)(x * h + dYs[0][i] * Rr[r]);
            gy[f * ld + p] = (T)(y * h + dYs[1][i] * Rr[r]);
            gz[f * ld + p] = (T)(z * h + dYs[2][i] * Rr[r]);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// K1: basis functions of the shells of one angular momentum L on a chunk of
// points.  grid = (chunk/128, shells of this L), block = 128 points; the
// shell's exponents, norms and contraction matrix are staged in shared
// memory first (global memory for shells larger than the staging area).
// ---------------------------------------------------------------------------
constexpr int kStagePrim = 64;
constexpr int kStageCon = 512;

template <int L, bool GRAD, typename T>
__global__ void __launch_bounds__(128) k_basis_l(const DevShell* __restrict__ shells, const int* __restrict__ ids,
                                                 const double* __restrict__ atoms, const double* __restrict__ exps,
                                                 const double* __restrict__ norms, const double* __restrict__ contr,
                                                 DevSA sa, const double* __restrict__ px, const double* __restrict__ py,
                                                 const double* __restrict__ pz, int64_t p0, int64_t nvalid, int64_t ld,
                                                 T* __restrict__ phi, T* __restrict__ gx, T* __restrict__ gy,
                                                 T* __restrict__ gz) {
  __shared__ double s_exp[kStagePrim], s_nrm[kStagePrim], s_con[kStageCon];
  DevShell S = shells[ids[blockIdx.y]];
  const double *e_src = exps + S.exp_off, *n_src = norms + S.exp_off, *c_src = contr + S.con_off;
  const bool staged = S.nexp <= kStagePrim && S.nexp * S.ncontr <= kStageCon;
  if (staged) {
    for (int i = threadIdx.x; i < S.nexp; i += blockDim.x) {
      s_exp[i] = e_src[i];
      s_nrm[i] = n_src[i];
    }
    for (int i = threadIdx.x; i < S.nexp * S.ncontr; i += blockDim.x) s_con[i] = c_src[i];
    __syncthreads();
    S.exp_off = 0;
    S.con_off = 0;
  }
  const int64_t p = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (p >= ld) return;
  const bool valid = p < nvalid;
  double x = 0, y = 0, z = 0;
  if (valid) {
    x = px[p0 + p] - atoms[3 * S.atom];
    y = py[p0 + p] - atoms[3 * S.atom + 1];
    z = pz[p0 + p] - atoms[3 * S.atom + 2];
  }
  shell_at_point<L, GRAD, T, double>(S, sa, x, y, z, staged ? s_exp : exps, staged ? s_nrm : norms,
                                     staged ? s_con : contr, valid, p, ld, phi, gx, gy, gz);
}

}  // namespace pgxc
