// kernels.h -- host-side launch interface between the C ABI and the kernels.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "pgxc_common.cuh"
#include "xc_functional.cuh"

namespace pgxc {

// Device pointers and sizes of one context, passed to every launcher.
struct BuildArgs {
  // basis
  const DevShell* shells = nullptr;
  int nshells = 0;
  const int* shl[kMaxL + 1] = {};  // shell indices of each angular momentum
  int nshl[kMaxL + 1] = {};
  const double* atoms = nullptr;
  const double* exps = nullptr;
  const double* norms = nullptr;
  const double* contr = nullptr;
  const int2* rng = nullptr;       // [lo, hi) primitive range of each contraction of segmented shells
  DevSA sa;
  XcConst xc;
  // grid (SoA, whole grid)
  const double* px = nullptr;
  const double* py = nullptr;
  const double* pz = nullptr;
  const double* w = nullptr;
  // chunk work arrays, [function][ldp]
  int64_t ldp = 0;      // points per chunk (multiple of 64)
  double* phi = nullptr;
  double* gx = nullptr;
  double* gy = nullptr;
  double* gz = nullptr;
  double* Z = nullptr;
  // per-point arrays [ldp]
  double* rho = nullptr;
  double* grx = nullptr;
  double* gry = nullptr;
  double* grz = nullptr;
  double* A = nullptr;
  double* Bx = nullptr;
  double* By = nullptr;
  double* Bz = nullptr;
  double* partial = nullptr;  // 2 per functional block
  double* acc = nullptr;      // {E, cE, N, cN}
  // density matrix
  int64_t ldc = 0;            // nbas padded to 64
  double* C = nullptr;        // [nocc_pad][ldc]
  double* Cocc = nullptr;
  const double* occ = nullptr;
  double* P = nullptr;        // [ldc][ldc]
  // potential tiles
  int nt = 0;                 // ldc / 64
  int ntiles = 0;             // nt (nt + 1) / 2
  int nsplit = 0;
  int64_t kspan = 0;          // points per split (multiple of 16)
  const int2* tiles = nullptr;
  const int* tile_of = nullptr;
  double* vpart = nullptr;    // [nsplit][ntiles][64*64]
};

void launch_basis_f64(const BuildArgs& a, int64_t p0, int64_t nvalid, bool grad, cudaStream_t st);
// basis values (and gradients) of every shell at points [p0, p0+ld) of (px,py,pz), FP64, [f][ld] layout
void launch_basis(const BuildArgs& a, const double* px, const double* py, const double* pz, int64_t p0,
                  int64_t nvalid, int64_t ld, double* phi, double* gx, double* gy, double* gz, cudaStream_t st);
void launch_basis_points_f64(const BuildArgs& a, const double* px, const double* py, const double* pz, int64_t n,
                             int64_t ld, double* phi, double* gx, double* gy, double* gz, cudaStream_t st);
void launch_pmat_f64(const BuildArgs& a, int64_t kpad, cudaStream_t st);
void launch_density_f64(const BuildArgs& a, bool gga, cudaStream_t st);
void launch_functional_f64(const BuildArgs& a, int64_t p0, int64_t nvalid, bool gga, cudaStream_t st);
// the functional on ntiles whole 128-point tiles, one partial pair per tile (no reduction)
void launch_functional_tiles(const BuildArgs& a, int64_t p0, int64_t ntiles, bool gga, cudaStream_t st);
// open shell: pa / pb = 8 point columns of ld per spin (rho, grad rho, A, B)
void launch_functional2_f64(const XcConst& K, const double* w, double* pa, double* pb, int64_t ld, int64_t p0,
                            int64_t nvalid, bool gga, double* partial, double* acc, cudaStream_t st);
// Fixed-order sum of nblocks {w f, w rho} block partials, Kahan-added into acc[4].
void launch_sum_partials(const double* partial, int nblocks, double* acc, cudaStream_t st);
// The meta-GGA functional step of the screened build (mgga.cu): pt as
// the screened point arrays (8 planes of ld per spin: rho, grad rho, A, B),
// tq 4 planes of ld per spin (the three 2 tau_j contractions, then C).
void launch_xc_points_mgga(int functional, int ispin, int64_t n, const double* rho, const double* gam, const double* tau, double* f,
                           double* fr, double* fg, double* ft, cudaStream_t st);
void launch_functional_mgga(int functional, int ispin, const double* w, double* pt, double* tq, int64_t ld, int64_t p0,
                            int64_t nvalid, double* partial, double* acc, cudaStream_t st);
void launch_zbuild_f64(const BuildArgs& a, bool gga, cudaStream_t st);
void launch_vpot_f64(const BuildArgs& a, bool gga, cudaStream_t st);
void launch_pack(const BuildArgs& a, int64_t nbas, int ispin, int spin, double* ham, cudaStream_t st);

// point-wise functional and Becke weights (standalone entry points)
void launch_xc_points(int functional, int ispin, int64_t n, const double* rho, const double* gam, double* f,
                      double* fr, double* fg, cudaStream_t st);
// Becke partition weights of n points (atom-atom distances into dist, natm^2);
// returns the launch status
cudaError_t launch_becke(const double* atoms, double* dist, int natm, const double* px, const double* py,
                         const double* pz, const int* owner, int64_t n, double* w, cudaStream_t st);
// message returned by pgxc_last_error(NULL)
void set_global_error(const std::string& msg);

void launch_scale_inplace(double* x, const double* s, int64_t n, cudaStream_t st);

}  // namespace pgxc
