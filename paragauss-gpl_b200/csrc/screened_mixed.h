// screened_mixed.h -- INT8 tensor-core (tcgen05 kind::i8, Ozaki split) stages
// of the screened XC build.  The FP64 basis, the functional and the packing are
// shared with the FP64 screened build (screened.cu).
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "kernels.h"

namespace pgxc {

struct ScreenMixed;

// One context of a multi-context set (screened.cu, screen_set_*): the
// tensor-core kernels take the density-matrix digits and the potential
// matrix of each tile's context from this table.
struct SetMolDev {
  const unsigned long long* P8;  // digits of P, [nbas][nbas]
  const int* e_P;                // row scales of P
  int64_t nbas;
  double* V;                     // potential accumulator, [nbas][ldv]
  int64_t ldv;
};

struct ScreenMixedInput {
  int64_t nbas = 0, ldc = 0;
  bool gga = false;
  int nspin = 1;             // density matrices kept in digit form (2 for open shell)
  int64_t chunk_slots = 0;   // slot rows of the chunk buffers (slack included)
  int64_t chunk_tiles = 0;
  int max_n = 0;             // largest padded slot count of a tile
  int64_t chunk_bstages = 0; // density B stages of the largest chunk
  const int64_t* b_off = nullptr;  // device [ntiles + 1]: first density B stage of each tile
  // resident point digits (basis kept across builds): slot rows and tiles of the whole grid, 0 -> per chunk
  int64_t resident_slots = 0, resident_tiles = 0;
};

// device bytes per slot row and per tile of the chunk buffers
int64_t screen_mixed_bytes_per_slot();
int64_t screen_mixed_bytes_per_tile();
// density B stages (48-slot blocks x 32-slot K steps) of a tile with n slots, and bytes per stage
int64_t screen_mixed_bstages(int64_t n);
int64_t screen_mixed_bytes_per_bstage();
int screen_mixed_create(ScreenMixed** out, const ScreenMixedInput& in, std::string& err);
void screen_mixed_destroy(ScreenMixed* m);
// INT8 digits of the FP64 density matrix P of spin `spin` (per-row scales); returns launches
int screen_mixed_prepare(ScreenMixed* m, const double* P, int64_t ldc, int spin, cudaStream_t st);
// Operands of the density contraction: INT8 digits of phi (per-point scales
// from pmax, the bit patterns of the largest |phi| of each point of the
// chunk) and the gathered digits of P[S_t, S_t] of every tile (spin 0)
// so / to: the chunk's first slot / tile in the resident digit arrays (0 when they are per chunk)
int screen_mixed_basis(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                       const double* phi, const unsigned long long* pmax, int64_t so, int64_t to, cudaStream_t st,
                       const int* tile_mol = nullptr, const SetMolDev* mols = nullptr);
// the functional kind of the following launches (a set's chunks alternate)
void screen_mixed_set_gga(ScreenMixed* m, bool gga);
// the gathered digits of P_spin[S_t, S_t] of every tile (replaces the previous spin's);
// with tile_mol, tile t's digits come from mols[tile_mol[t]] instead
int screen_mixed_gather(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                        int spin, cudaStream_t st, const int* tile_mol = nullptr, const SetMolDev* mols = nullptr);
int screen_mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                         const double* phi, const double* gx, const double* gy, const double* gz, double* rho,
                         double* grx, double* gry, double* grz, int64_t so, int64_t to, cudaStream_t st);
// the same with 32-bit gradient planes (the INT8 build's basis values: phi in
// FP64, grad phi in FP32)
int screen_mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                         const double* phi, const float* gx, const float* gy, const float* gz, double* rho,
                         double* grx, double* gry, double* grz, int64_t so, int64_t to, cudaStream_t st);
// Z digits (per-slot scales), then H[S_t, S_t] += Z_t^T phi_t scatter-added into V;
// records k0 / k1 around the contraction kernel
// (with tile_mol: into mols[tile_mol[t]].V of each tile t instead of V)
int screen_mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, const int* slot_tile, int64_t t0,
                           int64_t nt, int64_t s0, int64_t ns, const double* phi, const double* gx, const double* gy,
                           const double* gz, const double* A, const double* Bx, const double* By, const double* Bz,
                           double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1,
                           const int* tile_mol = nullptr, const SetMolDev* mols = nullptr);
int screen_mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, const int* slot_tile, int64_t t0,
                           int64_t nt, int64_t s0, int64_t ns, const double* phi, const float* gx, const float* gy,
                           const float* gz, const double* A, const double* Bx, const double* By, const double* Bz,
                           double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1,
                           const int* tile_mol = nullptr, const SetMolDev* mols = nullptr);
// the digits of P_spin and their row scales (read by a set's gather)
void screen_mixed_p8(ScreenMixed* m, int spin, const unsigned long long** P8, const int** e_P);
// copies the device error flag (a bounded wait ran out) to *flag and clears it
int screen_mixed_error_flag(ScreenMixed* m, cudaStream_t st, int* flag);

}  // namespace pgxc
