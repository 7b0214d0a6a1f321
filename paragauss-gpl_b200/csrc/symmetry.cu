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

}  // namespace

void launch_sym_orbitals(const SymDev& S, const double* Csa, const int64_t* cofs, const int* nocc,
                         const int64_t* col0, int nocc_max, double* C, int64_t ldc, cudaStream_t st) {
  if (S.ngroups == 0 || nocc_max == 0) return;
  const int threads = nocc_max >= 128 ? 128 : ((nocc_max + 31) / 32) * 32;
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
