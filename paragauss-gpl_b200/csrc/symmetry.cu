// symmetry.cu -- the two gathers of the symmetry-adapted build (symmetry.h).
//
// Both are small next to the build: each C1 row or SA column of U holds at
// most the order of the group entries, so the orbital gather reads
// (listed entries) x nocc values and the potential gather reads
// sum_i np_i dims_i^2 (entries per column)^2 values of V.
#include <cmath>

#include "symmetry.h"

namespace pgxc {

namespace {

__global__ void k_sym_orbitals(SymDev S, const double* __restrict__ Csa, const int64_t* __restrict__ cofs,
                               const int* __restrict__ nocc, const int64_t* __restrict__ col0,
                               double* __restrict__ C, int64_t ldc) {
  const int g = blockIdx.x;
  const int ip = S.grp_ip[g];
  const int a = S.grp_ao[g];
  const int irr = S.ip_irrep[ip];
  const int n = nocc[irr];
  const int dim = S.dims[irr];
  const double* Ci = Csa + cofs[irr];
  const int64_t e0 = S.grp_ptr[g], e1 = S.grp_ptr[g + 1];
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double s = 0.0;
    for (int64_t e = e0; e < e1; ++e) s += S.row_coef[e] * Ci[S.row_fn[e] + (int64_t)dim * k];
    C[a + ldc * (col0[ip] + k)] = s;
  }
}

__device__ __forceinline__ int64_t packed(int64_t a, int64_t b) {
  const int64_t hi = a > b ? a : b, lo = a > b ? b : a;
  return hi * (hi + 1) / 2 + lo;
}

__global__ void k_sym_potential(SymDev S, int ispin, const double* __restrict__ V, double* __restrict__ H) {
  const int irr = blockIdx.y;
  const int64_t dim = S.dims[irr];
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= dim * (dim + 1) / 2) return;
  // t = g (g + 1) / 2 + f with f <= g
  int64_t g = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (g * (g + 1) / 2 > t) --g;
  while ((g + 1) * (g + 2) / 2 <= t) ++g;
  const int64_t f = t - g * (g + 1) / 2;
  const int np = S.partners[irr];
  for (int s = 0; s < ispin; ++s) {
    double sum = 0.0;
    for (int p = 0; p < np; ++p) {
      const int ip = S.ipbase[irr] + p;
      const int64_t cf = S.colbase[ip] + f, cg = S.colbase[ip] + g;
      for (int64_t i = S.col_ptr[cf]; i < S.col_ptr[cf + 1]; ++i) {
        const int64_t a = S.col_ao[i];
        const double ca = S.col_coef[i];
        double r = 0.0;
        for (int64_t j = S.col_ptr[cg]; j < S.col_ptr[cg + 1]; ++j)
          r += S.col_coef[j] * V[s + ispin * packed(a, S.col_ao[j])];
        sum += ca * r;
      }
    }
    H[s + ispin * (S.pkofs[irr] + t)] = sum / np;
  }
}

// One thread per element quadruple of a pseudo-2D irrep's packed matrix.
// Pair q: blocks X (first function px, half hx) >= Y (py, hy) of one irrep
// (packed offset pk); element (r, c) of the pair's A x A part, r < hx, c < hy
// (X == Y: c <= r).  The reference's loops (xc_pseudo2d_sym,
// modules/xc_hamiltonian.f90:2637-2779) touch every element of a quadruple
// once, so the quadruples are independent.
__device__ __forceinline__ int64_t pk1(int64_t j, int64_t k) { return j * (j + 1) / 2 + k; }  // k <= j, 0-based

__global__ void k_pseudo2d(const Pseudo2dPair* __restrict__ pairs, const int64_t* __restrict__ first,
                           int64_t npairs_total, int ispin, double* __restrict__ ham) {
  // first[q] = the pair's first quadruple; quadruples of pair q: [first[q], first[q + 1])
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < first[npairs_total];
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = npairs_total;  // the pair holding quadruple e
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (first[mid] <= e) lo = mid;
      else hi = mid;
    }
    const Pseudo2dPair P = pairs[lo];
    const int64_t t = e - first[lo];
    int64_t r, c;
    if (P.same) {  // t enumerates (r, c), c <= r
      r = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while (r * (r + 1) / 2 > t) --r;
      while ((r + 1) * (r + 2) / 2 <= t) ++r;
      c = t - r * (r + 1) / 2;
    } else {
      r = t / P.hy;
      c = t - r * P.hy;
    }
    for (int s = 0; s < ispin; ++s) {
      auto at = [&](int64_t j, int64_t k) -> double& { return ham[s + ispin * (P.pk + pk1(j, k))]; };
      if (P.same) {
        // A x A and B x B (r >= c): their mean into both
        double& aa = at(P.px + r, P.px + c);
        double& bb = at(P.px + P.hx + r, P.px + P.hx + c);
        aa = 0.5 * (aa + bb);
        bb = aa;
        // B x A: H(B_c, A_r) = (H(B_c, A_r) - H(B_r, A_c)) / 2, H(B_r, A_c) = -H(B_c, A_r)
        double& x4 = at(P.px + P.hx + c, P.px + r);
        double& x3 = at(P.px + P.hx + r, P.px + c);
        x4 = 0.5 * (x4 - x3);
        x3 = -x4;
      } else {
        double& aa = at(P.px + r, P.py + c);
        double& bb = at(P.px + P.hx + r, P.py + P.hy + c);
        aa = 0.5 * (aa + bb);
        bb = aa;
        double& ab = at(P.px + r, P.py + P.hy + c);
        double& ba = at(P.px + P.hx + r, P.py + c);
        ab = 0.5 * (ab - ba);
        ba = -ab;
      }
    }
  }
}

}  // namespace

void launch_sym_orbitals(const SymDev& S, const double* Csa, const int64_t* cofs, const int* nocc,
                         const int64_t* col0, int nocc_max, double* C, int64_t ldc, cudaStream_t st) {
  if (S.ngroups == 0 || nocc_max == 0) return;
  const int threads = 128;  // whole groups of four warps (kBlock4); threads past nocc idle
  k_sym_orbitals<<<S.ngroups, threads, 0, st>>>(S, Csa, cofs, nocc, col0, C, ldc);
}

void launch_sym_potential(const SymDev& S, int max_dim, int ispin, const double* V, double* ham_sym,
                          cudaStream_t st) {
  const int64_t np_max = (int64_t)max_dim * (max_dim + 1) / 2;
  if (np_max == 0 || S.n_irrep == 0) return;
  const dim3 grid((unsigned)((np_max + 255) / 256), (unsigned)S.n_irrep);
  k_sym_potential<<<grid, 256, 0, st>>>(S, ispin, V, ham_sym);
}

}  // namespace pgxc

namespace pgxc {

void launch_pseudo2d(const Pseudo2dPair* pairs, const int64_t* first, int64_t npairs, int64_t nquads, int ispin,
                     double* ham, cudaStream_t st) {
  if (npairs == 0 || nquads == 0) return;
  const unsigned nb = (unsigned)std::min<int64_t>((nquads + 255) / 256, 148 * 16);
  k_pseudo2d<<<nb, 256, 0, st>>>(pairs, first, npairs, ispin, ham);
}

}  // namespace pgxc
