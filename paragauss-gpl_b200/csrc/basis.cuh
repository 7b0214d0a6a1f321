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
// All arithmetic is FP64 in both precision modes.
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
// (radial0/radial1, modules/orbital_module.f90:1823-1854).
__device__ __forceinline__ double prim_value(double alpha, double norm, double r2) {
  const double ar2 = alpha * r2;
  return ar2 < 50.0 ? norm * exp(-ar2) : 0.0;
}

// Evaluate the selected radial functions of one shell at one point.  The
// selected radial indices are the set bits of `mask` (nsel of them, in
// increasing order); selected function k of independent function i is stored
// at row base + i*nsel + k, column p of the [row][ld] arrays.  The dense
// layout is mask = all nrad bits, base = S.f0 (row = function index); the
// screened layout is the tile's significant radial functions and their slot.
// exps/norms/contr/rng may point to shared memory (plain loads); rng is the
// shell's [lo, hi) primitive range per contraction (used when S.seg).
template <int L, bool GRAD>
__device__ __forceinline__ void shell_at_point(const DevShell& S, const DevSA& sa, double x, double y, double z,
                                               const double* exps, const double* norms, const double* contr,
                                               const int2* rng, bool valid, uint64_t mask, int64_t base, int nsel,
                                               int64_t p,
                                               int64_t ld, double* __restrict__ phi, double* __restrict__ gx,
                                               double* __restrict__ gy, double* __restrict__ gz, double& vmax) {
  double Y[16];
  double dY[3][16];
  solid_harmonics<L, double>(x, y, z, Y, dY);
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
  const double* ex = exps + S.exp_off;
  const double* nr = norms + S.exp_off;
  const double* cc = contr + S.con_off;
  if (S.seg) {
    // segmented contractions: each selected radial function sums only its own primitives
    uint64_t rem = mask;
    for (int k = 0; k < nsel; ++k) {
      const int rr = __ffsll((long long)rem) - 1;
      rem &= rem - 1;
      const int2 rg = rng[rr];
      double Rr = 0.0, dR = 0.0;
      if (valid) {
        for (int e = rg.x; e < rg.y; ++e) {
          const double alpha = ex[e];
          const double v = prim_value(alpha, nr[e], r2);
          const double cf = cc[e + (int64_t)S.nexp * rr];
          Rr += cf * v;
          dR += cf * ((-2.0 * alpha) * v);
        }
      }
#pragma unroll
      for (int i = 0; i < 2 * L + 1; ++i) {
        const int64_t f = base + (int64_t)i * nsel + k;
        phi[f * ld + p] = Ys[i] * Rr;
        vmax = fmax(vmax, fabs(Ys[i] * Rr));
        if (GRAD) {
          const double h = Ys[i] * dR;
          gx[f * ld + p] = x * h + dYs[0][i] * Rr;
          gy[f * ld + p] = y * h + dYs[1][i] * Rr;
          gz[f * ld + p] = z * h + dYs[2][i] * Rr;
        }
      }
    }
    return;
  }
  uint64_t rem = mask;
  for (int k0 = 0; k0 < nsel; k0 += kRadGroup) {
    int rr[kRadGroup];
#pragma unroll
    for (int r = 0; r < kRadGroup; ++r) {
      if (k0 + r < nsel) {
        rr[r] = __ffsll((long long)rem) - 1;
        rem &= rem - 1;
      } else {
        rr[r] = -1;
      }
    }
    double Rr[kRadGroup], dR[kRadGroup];
#pragma unroll
    for (int r = 0; r < kRadGroup; ++r) { Rr[r] = 0.0; dR[r] = 0.0; }
    if (valid) {
      for (int e = 0; e < S.nexp; ++e) {
        const double alpha = ex[e];
        const double v = prim_value(alpha, nr[e], r2);
        const double dv = (-2.0 * alpha) * v;
#pragma unroll
        for (int r = 0; r < kRadGroup; ++r) {
          if (rr[r] >= 0) {
            double cf;
            if (rr[r] < S.nunc) cf = (e == rr[r]) ? 1.0 : 0.0;
            else cf = cc[e + (int64_t)S.nexp * (rr[r] - S.nunc)];
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
        if (rr[r] >= 0) {
          const int64_t f = base + (int64_t)i * nsel + k0 + r;
          phi[f * ld + p] = Ys[i] * Rr[r];
          vmax = fmax(vmax, fabs(Ys[i] * Rr[r]));
          if (GRAD) {
            const double h = Ys[i] * dR[r];
            gx[f * ld + p] = x * h + dYs[0][i] * Rr[r];
            gy[f * ld + p] = y * h + dYs[1][i] * Rr[r];
            gz[f * ld + p] = z * h + dYs[2][i] * Rr[r];
          }
        }
      }
    }
  }
}

// Stage one shell's exponents, norms and contraction matrix in shared memory
// (when they fit); returns the pointers to use.
constexpr int kStagePrim = 64;
constexpr int kStageCon = 512;
struct ShellStage {
  double e[kStagePrim], n[kStagePrim], c[kStageCon];
  int2 r[64];
};
// Stages the shell (when it fits) and its contraction ranges; returns the
// range pointer to use (shared memory).
__device__ __forceinline__ bool stage_shell(ShellStage& st, DevShell& S, const double* exps, const double* norms,
                                            const double* contr, const int2* rng) {
  const bool staged = S.nexp <= kStagePrim && S.nexp * S.ncontr <= kStageCon;
  if (staged) {
    const double *e_src = exps + S.exp_off, *n_src = norms + S.exp_off, *c_src = contr + S.con_off;
    for (int i = threadIdx.x; i < S.nexp; i += blockDim.x) {
      st.e[i] = e_src[i];
      st.n[i] = n_src[i];
    }
    for (int i = threadIdx.x; i < S.nexp * S.ncontr; i += blockDim.x) st.c[i] = c_src[i];
    S.exp_off = 0;
    S.con_off = 0;
  }
  if (S.seg)
    for (int i = threadIdx.x; i < S.nrad; i += blockDim.x) st.r[i] = rng[S.rad_off + i];
  __syncthreads();
  return staged;
}

__host__ __device__ constexpr uint64_t all_radial(int nrad) { return nrad >= 64 ? ~0ull : ((1ull << nrad) - 1); }

// ---------------------------------------------------------------------------
// K1 (dense): basis functions of the shells of one angular momentum L on a
// chunk of points.  grid = (chunk/128, shells of this L), block = 128 points.
// ---------------------------------------------------------------------------
template <int L, bool GRAD>
__global__ void __launch_bounds__(128) k_basis_l(const DevShell* __restrict__ shells, const int* __restrict__ ids,
                                                 const double* __restrict__ atoms, const double* __restrict__ exps,
                                                 const double* __restrict__ norms, const double* __restrict__ contr,
                                                 const int2* __restrict__ rng, DevSA sa, const double* __restrict__ px,
                                                 const double* __restrict__ py,
                                                 const double* __restrict__ pz, int64_t p0, int64_t nvalid, int64_t ld,
                                                 double* __restrict__ phi, double* __restrict__ gx,
                                                 double* __restrict__ gy, double* __restrict__ gz) {
  __shared__ ShellStage st;
  DevShell S = shells[ids[blockIdx.y]];
  const bool staged = stage_shell(st, S, exps, norms, contr, rng);
  const int64_t p = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (p >= ld) return;
  const bool valid = p < nvalid;
  double x = 0, y = 0, z = 0;
  if (valid) {
    x = px[p0 + p] - atoms[3 * S.atom];
    y = py[p0 + p] - atoms[3 * S.atom + 1];
    z = pz[p0 + p] - atoms[3 * S.atom + 2];
  }
  double vmax = 0.0;
  shell_at_point<L, GRAD>(S, sa, x, y, z, staged ? st.e : exps, staged ? st.n : norms, staged ? st.c : contr, st.r,
                          valid, all_radial(S.nrad), S.f0, S.nrad, p, ld, phi, gx, gy, gz, vmax);
}

// ---------------------------------------------------------------------------
// K1 (screened): a work item is the significant radial functions of one shell
// on the 128 points of one tile.  Rows are slots of the chunk's compact
// [slot][128] arrays (slot - s0); with pmax, the largest |phi| of each point
// of the chunk (tile - t0) is max-reduced into it.
//
// An item carries every field its evaluation needs (atom position, primitive
// and contraction offsets), so that the loads of the next items do not depend
// on one another.  A block walks a contiguous range of items; each warp keeps
// the item records lane-distributed (lane k holds 32-bit word k) two items
// ahead, and the current item's exponents and norms in lanes (lane e holds
// primitive e), broadcast with shuffles.  Consecutive items of a tile reuse
// the point coordinates.
// ---------------------------------------------------------------------------
struct BasisItem {
  double ax, ay, az;        // words 0-5: atom position
  int64_t slot;             // 6-7: global slot of the shell's first significant function
  unsigned long long mask;  // 8-9: significant radial functions of the shell
  int tile;                 // 10: global tile index
  int nsig;                 // 11: popcount(mask)
  int exp_off;              // 12: into exponents / norms
  int con_off;              // 13: into contractions (nexp x ncontr column-major)
  int rad_off;              // 14: into the radial-range table (seg shells)
  int nexp;                 // 15
  int nunc;                 // 16
  int seg;                  // 17
  int pad_[2];
};
static_assert(sizeof(BasisItem) == 80, "BasisItem is read as 20 words");
constexpr int kItemWords = 20;

__device__ __forceinline__ int item_i(unsigned w, int k) { return (int)__shfl_sync(0xffffffffu, w, k); }
__device__ __forceinline__ double item_d(unsigned w, int k) {
  const unsigned lo = __shfl_sync(0xffffffffu, w, k), hi = __shfl_sync(0xffffffffu, w, k + 1);
  return __hiloint2double((int)hi, (int)lo);
}
__device__ __forceinline__ unsigned long long item_u64(unsigned w, int k) {
  const unsigned lo = __shfl_sync(0xffffffffu, w, k), hi = __shfl_sync(0xffffffffu, w, k + 1);
  return ((unsigned long long)hi << 32) | lo;
}

// GT: the element type of the gradient planes (double; float in the INT8
// build, whose potential and density gradient tolerate 24-bit gradients).
// Blocks per SM: with gradients 6, 5, 4, 4 for l = 0..3 (at most 80, 96, 128
// and 128 registers), without them 8, 8, 8, 7.  Without a bound the f-shell
// kernel took 164 registers and ran three blocks per SM, the slower form for
// the 500-atom grid; a bound of one block lets the compiler take 144-188
// registers for l <= 2, which cost the 60-atom build 0.6 ms.
template <int L, bool GRAD>
constexpr int basis_blocks() {
  return GRAD ? (L == 0 ? 6 : (L == 1 ? 5 : 4)) : (L <= 2 ? 8 : 7);
}
template <int L, bool GRAD, typename GT = double>
__global__ void __launch_bounds__(128, (basis_blocks<L, GRAD>())) k_basis_items(const BasisItem* __restrict__ items, int64_t nitems,
                                                     const double* __restrict__ exps, const double* __restrict__ norms,
                                                     const double* __restrict__ contr,
                                                     const int2* __restrict__ rng, DevSA sa,
                                                     const double* __restrict__ qx, const double* __restrict__ qy,
                                                     const double* __restrict__ qz, int64_t s0, int64_t t0,
                                                     double* __restrict__ phi, GT* __restrict__ gx,
                                                     GT* __restrict__ gy, GT* __restrict__ gz,
                                                     unsigned long long* __restrict__ pmax) {
  const int lane = threadIdx.x & 31;
  const int64_t per = (nitems + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(nitems, i0 + per);
  if (i0 >= i1) return;
  const unsigned* words = reinterpret_cast<const unsigned*>(items);
  auto load_item = [&](int64_t i) -> unsigned {
    return lane < kItemWords ? __ldg(words + min(i, i1 - 1) * kItemWords + lane) : 0u;
  };
  unsigned wc = load_item(i0), wn = load_item(i0 + 1);
  int nexp = item_i(wc, 15), eoff = item_i(wc, 12);
  double pe = 0.0, pn = 0.0;  // lane e: exponent and norm of primitive e of the current item
  if (lane < nexp) { pe = __ldg(exps + eoff + lane); pn = __ldg(norms + eoff + lane); }
  int tile = item_i(wc, 10);
  double px = __ldg(qx + (int64_t)tile * 128 + threadIdx.x);
  double py = __ldg(qy + (int64_t)tile * 128 + threadIdx.x);
  double pz = __ldg(qz + (int64_t)tile * 128 + threadIdx.x);
  double tmax = 0.0;
  for (int64_t i = i0; i < i1; ++i) {
    // loads for the next items, issued ahead of this item's arithmetic
    const unsigned wnn = load_item(i + 2);
    const int n_nexp = item_i(wn, 15), n_eoff = item_i(wn, 12), n_tile = item_i(wn, 10);
    double ne = 0.0, nn = 0.0;
    if (lane < n_nexp) { ne = __ldg(exps + n_eoff + lane); nn = __ldg(norms + n_eoff + lane); }
    double nx = px, ny = py, nz = pz;
    if (n_tile != tile) {
      const int64_t qn = (int64_t)n_tile * 128 + threadIdx.x;
      nx = __ldg(qx + qn); ny = __ldg(qy + qn); nz = __ldg(qz + qn);
    }
    // this item
    {
      const double x = px - item_d(wc, 0), y = py - item_d(wc, 2), z = pz - item_d(wc, 4);
      const int64_t base = (int64_t)item_u64(wc, 6) - s0;
      const uint64_t mask = item_u64(wc, 8);
      const int nsel = item_i(wc, 11), coff = item_i(wc, 13), roff = item_i(wc, 14), nunc = item_i(wc, 16);
      const bool seg = item_i(wc, 17) != 0;
      double Y[16];
      double dY[3][16];
      solid_harmonics<L, double>(x, y, z, Y, dY);
      const double r2 = x * x + y * y + z * z;
      double Ys[2 * L + 1], dYs[3][2 * L + 1];
#pragma unroll
      for (int k = 0; k < 2 * L + 1; ++k) {
        if (sa.identity) {
          Ys[k] = Y[L * L + k];
#pragma unroll
          for (int c = 0; c < 3; ++c) dYs[c][k] = dY[c][L * L + k];
        } else {
          double v = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
          for (int m = 0; m < 2 * L + 1; ++m) {
            const double cf = sa.c[L][k][m];
            v += cf * Y[L * L + m];
            g0 += cf * dY[0][L * L + m];
            g1 += cf * dY[1][L * L + m];
            g2 += cf * dY[2][L * L + m];
          }
          Ys[k] = v; dYs[0][k] = g0; dYs[1][k] = g1; dYs[2][k] = g2;
        }
      }
      // primitive e's exponent and norm: from lane e, or memory past 32 primitives
      auto prim = [&](int e, double& alpha, double& nrm) {
        if (e < 32) {
          alpha = __shfl_sync(0xffffffffu, pe, e);
          nrm = __shfl_sync(0xffffffffu, pn, e);
        } else {
          alpha = __ldg(exps + eoff + e);
          nrm = __ldg(norms + eoff + e);
        }
      };
      double vmax = 0.0;
      auto store = [&](int64_t f, double Rv, double dRv, int k) {
        const int64_t o = f * 128 + threadIdx.x;
        phi[o] = Ys[k] * Rv;
        vmax = fmax(vmax, fabs(Ys[k] * Rv));
        if (GRAD) {
          const double h = Ys[k] * dRv;
          gx[o] = (GT)(x * h + dYs[0][k] * Rv);
          gy[o] = (GT)(y * h + dYs[1][k] * Rv);
          gz[o] = (GT)(z * h + dYs[2][k] * Rv);
        }
      };
      if (seg) {
        // segmented contractions: each selected radial function sums only its own primitives
        uint64_t rem = mask;
        for (int k = 0; k < nsel; ++k) {
          const int rr = __ffsll((long long)rem) - 1;
          rem &= rem - 1;
          const int2 rg = __ldg(rng + roff + rr);
          double Rr = 0.0, dR = 0.0;
          for (int e = rg.x; e < rg.y; ++e) {
            double alpha, nrm;
            prim(e, alpha, nrm);
            const double v = prim_value(alpha, nrm, r2);
            const double cf = __ldg(contr + coff + e + (int64_t)nexp * rr);
            Rr += cf * v;
            dR += cf * ((-2.0 * alpha) * v);
          }
#pragma unroll
          for (int k2 = 0; k2 < 2 * L + 1; ++k2) store(base + (int64_t)k2 * nsel + k, Rr, dR, k2);
        }
      } else {
        uint64_t rem = mask;
        for (int k0 = 0; k0 < nsel; k0 += kRadGroup) {
          int rr[kRadGroup];
#pragma unroll
          for (int r = 0; r < kRadGroup; ++r) {
            if (k0 + r < nsel) {
              rr[r] = __ffsll((long long)rem) - 1;
              rem &= rem - 1;
            } else {
              rr[r] = -1;
            }
          }
          double Rr[kRadGroup], dR[kRadGroup];
#pragma unroll
          for (int r = 0; r < kRadGroup; ++r) { Rr[r] = 0.0; dR[r] = 0.0; }
          for (int e = 0; e < nexp; ++e) {
            double alpha, nrm;
            prim(e, alpha, nrm);
            const double v = prim_value(alpha, nrm, r2);
            const double dv = (-2.0 * alpha) * v;
#pragma unroll
            for (int r = 0; r < kRadGroup; ++r) {
              if (rr[r] >= 0) {
                const double cf = rr[r] < nunc ? (e == rr[r] ? 1.0 : 0.0)
                                               : __ldg(contr + coff + e + (int64_t)nexp * (rr[r] - nunc));
                Rr[r] += cf * v;
                dR[r] += cf * dv;
              }
            }
          }
#pragma unroll
          for (int k = 0; k < 2 * L + 1; ++k) {
#pragma unroll
            for (int r = 0; r < kRadGroup; ++r)
              if (rr[r] >= 0) store(base + (int64_t)k * nsel + k0 + r, Rr[r], dR[r], k);
          }
        }
      }
      // largest |phi| of each point over the tile's functions, max-reduced once per run of
      // items of one tile (non-negative doubles order like their bits)
      tmax = fmax(tmax, vmax);
      if (pmax && (n_tile != tile || i + 1 == i1)) {
        atomicMax(pmax + ((int64_t)tile - t0) * 128 + threadIdx.x, (unsigned long long)__double_as_longlong(tmax));
        tmax = 0.0;
      }
    }
    wc = wn;
    wn = wnn;
    nexp = n_nexp;
    eoff = n_eoff;
    pe = ne;
    pn = nn;
    tile = n_tile;
    px = nx; py = ny; pz = nz;
  }
}

}  // namespace pgxc
