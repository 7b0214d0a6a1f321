// symmetry.h -- symmetry-adapted bases (n_irrep >= 1, partners >= 1) folded
// into the C1 build by two sparse gathers on the device.
//
// A symmetry-adapted function f of irrep i, partner p is phi_f = sum_a U[a,f]
// chi_a over the context's C1 functions chi_a (the reference's symadapt
// coefficients over equal atoms, orbital_module.f90:2421-2619).  Then
//   rho = sum_i sum_p sum_k occ_ik / np_i (phi C_i)_k^2        (density_calc_nl)
//       = the C1 density of the orbitals U_ip C_i with occupations occ_i / np_i,
//   V_i = 1/np_i sum_p phi_p^T v phi_p = 1/np_i sum_p U_ip^T V_C1 U_ip
// (calc_xcks integrate / calc_xcks_nl, modules/xc_hamiltonian.f90:987-1034,
// :1455-1566), on any grid, the symmetry-reduced one of the reference included.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pgxc {

// Device tables of one symmetry adaptation (sorted copies of U).
struct SymDev {
  int n_irrep = 0;
  const int* dims = nullptr;      // [n_irrep]
  const int* partners = nullptr;  // [n_irrep]
  const int* ipbase = nullptr;    // [n_irrep] first (irrep, partner) index of each irrep
  const int64_t* pkofs = nullptr; // [n_irrep] packed-triangle offset of each irrep
  const int* ip_irrep = nullptr;  // [nip] irrep of each (irrep, partner)
  int ngroups = 0;                // (ip, C1 function) groups of U rows
  const int* grp_ip = nullptr;
  const int* grp_ao = nullptr;
  const int64_t* grp_ptr = nullptr;  // [ngroups + 1] into row_fn / row_coef
  const int* row_fn = nullptr;
  const double* row_coef = nullptr;
  const int64_t* colbase = nullptr;  // [nip] first column index of each (irrep, partner)
  const int64_t* col_ptr = nullptr;  // [ncol + 1] into col_ao / col_coef
  const int* col_ao = nullptr;
  const double* col_coef = nullptr;
};

// C_C1[a + ldc (col0[ip] + k)] = sum_{f in row (ip, a)} U[a,f] C_i[f + dims_i k]
// for one spin; Csa holds the irreps' orbitals of that spin at cofs[i]
// (dims_i x nocc_i column-major), nocc[i] per irrep, col0[ip] the first
// column of each (irrep, partner) block.
void launch_sym_orbitals(const SymDev& S, const double* Csa, const int64_t* cofs, const int* nocc,
                         const int64_t* col0, int nocc_max, double* C, int64_t ldc, cudaStream_t st);

// ham_sym[s + ispin (pkofs[i] + t)] = 1/np_i sum_p sum_{a in col (ip,f)} sum_{b in col (ip,g)}
// U[a,f] U[b,g] V[s + ispin (hi (hi+1)/2 + lo)], t the packed index of f <= g.
void launch_sym_potential(const SymDev& S, int max_dim, int ispin, const double* V, double* ham_sym,
                          cudaStream_t st);

// Pseudo-2D irreps (xc_pseudo2d_sym, modules/xc_hamiltonian.f90:2637-2779):
// the functions of every (unique atom, l) block of such an irrep come in two
// halves A, B; the matrix is made to satisfy H(X_A, Y_A) = H(X_B, Y_B) and
// H(X_A, Y_B) = -H(X_B, Y_A) for every pair of blocks X >= Y.  One entry per
// block pair: X's first function px and half hx, Y's py, hy (0-based within
// the irrep), the irrep's packed offset pk, same = (X == Y).
struct Pseudo2dPair {
  int64_t pk;
  int64_t px, hx, py, hy;
  int64_t same;
};
// first[q]: quadruples before pair q (first[npairs] = nquads)
void launch_pseudo2d(const Pseudo2dPair* pairs, const int64_t* first, int64_t npairs, int64_t nquads, int ispin,
                     double* ham, cudaStream_t st);

}  // namespace pgxc
