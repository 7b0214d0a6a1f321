// gradient.h -- post-SCF XC nuclear gradient on the device.
//
// dE_xc/dR_A of E_xc = sum_g w_g f(rho(r_g), gamma(r_g)) with the grid
// attached to the atoms (r_g = R_host + fixed offset) and w_g = w_raw(g)
// W_host(r_g), the Becke weight of the host atom: the derivative of the
// discrete energy the build integrates, as the reference's post-SCF
// gradients with moving grid and weight gradients (post_scf_module.f90
// :2930-3060, density_calc_ph_nl, grid_module.f90 becke1).
//
// With X^s = Phi P^s and Y^s_j = d_j Phi P^s (per chunk of points),
//   q^s_mu,k(g) = 2 [a_s d_k phi_mu X^s_mu + sum_j b_sj (d_k d_j phi_mu X^s_mu + d_k phi_mu Y^s_j,mu)],
// a_s = w df/drho_s and b_s = w (2 df/dgamma_ss grad rho_s + df/dgamma_ab grad rho_s'), the
// orbital terms are  -sum_g q_mu(g) to atom(mu)  and  +sum_mu q_mu(g) to host(g);
// the weight term is sum_g w_raw f dW_host(r_g)/dR.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace pgxc {

// Basis values, gradients and Hessians of every function on points
// [p0, p0 + nvalid) of the context's grid: out[c * plane + f * ld + p],
// c = 0 phi, 1..3 d/dx, d/dy, d/dz, 4..9 xx, xy, xz, yy, yz, zz.
void launch_basis_hess(const BuildArgs& a, int64_t p0, int64_t nvalid, int64_t ld, int64_t plane, double* out,
                       cudaStream_t st);

// Per point of the chunk: rho_s, grad rho_s (and for meta-GGAs tau_s) from X,
// Y and the basis values, the functional, and the coefficients a_s, b_s, c_s
// (coef[(5 s + c) ld + p]; c_s = w df/dtau_s, 0 below meta-GGAs) and
// ef = w_raw f; E_xc = sum w f is added into *exc.
// out[f][p] = sum_g basis_j[g][p] P[g][f], f < nbas, p < ld (ld a multiple of
// 64; basis_j followed by at least 15 more rows of ld; P ldc x ldc, zero past nbas)
void launch_grad_xy(const double* basis_j, int64_t ld, const double* P, int64_t ldc, int64_t nbas, double* out,
                    cudaStream_t st);
void launch_grad_points(const XcConst& K, int functional, bool gga, int ispin, int64_t nbas, int64_t ld, int64_t p0,
                        int64_t nvalid, const double* w, const double* wraw, const double* basis, int64_t plane,
                        const double* XY, double* coef, double* ef, double* exc, cudaStream_t st);

// GGAs (not meta-GGAs): W = sum_j b_j d_j phi of the chunk (coef_b: the three
// b planes of one spin), rows nbas .. round_up(nbas, 16) - 1 zero; the orbital
// terms then take V = W P (plane 2 of the spin) in place of the three Y_j.
void launch_grad_w(int64_t nbas, int64_t ld, const double* basis, int64_t plane, const double* coef_b, double* W,
                   cudaStream_t st);

// The orbital terms: -sum_g q to atom(mu) (fatom[mu]) and +sum_mu q to host(g).
void launch_grad_orbital(bool gga, bool mgga, int ispin, int64_t nbas, int64_t ld, int64_t p0, int64_t nvalid,
                         int natm, const int* fatom, const int* owner, const double* basis, int64_t plane,
                         const double* XY, const double* coef, double* grad, cudaStream_t st);

// The weight term sum_g ef_g dW_host(r_g)/dR over the chunk's points; dist is
// the natm x natm atom distance matrix followed by its reciprocals (the
// table of launch_becke); scratch holds 3.5 natm ld doubles.
void launch_grad_weights(const double* atoms, const double* dist, int natm, const double* px, const double* py,
                         const double* pz, const int* owner, int64_t p0, int64_t nvalid, int64_t ld, const double* ef,
                         double* scratch, double* grad, cudaStream_t st);

}  // namespace pgxc
