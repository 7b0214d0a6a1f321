// screened.h -- the screened (tile-sparse) XC build.
//
// The grid is reordered along a Morton curve and cut into tiles of 128 points
// (the reference's vla batches, made spatially compact).  For every tile the
// basis functions that can be nonzero on it are listed once per geometry;
// every per-cycle stage then works on the tile's compact [slot][128] block:
// the basis is evaluated only for listed functions, X = phi P_sig gathers the
// listed rows and columns of P, and V_sig = Z^T phi is scatter-added into V.
//
// A function is listed for a tile when, for some point of the tile,
//   threshold == 0: some primitive has alpha r^2 < 50 (the reference's own
//                   cutoff, modules/orbital_module.f90:1831-1854: every
//                   unlisted function is exactly zero on the tile);
//   threshold  > 0: in addition a bound on |phi| and |grad phi| reaches the
//                   threshold.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "kernels.h"

namespace pgxc {

struct ScreenPlan;

struct ScreenTimes {
  float basis = 0, density = 0, functional = 0, potential = 0, x = 0, v = 0;
  int64_t launches = 0;
};

// Host-side description of the context, for planning.
struct ScreenInput {
  const std::vector<DevShell>* shells;
  const double* atoms;        // host, 3 x natm
  int natm;
  int64_t nbas;
  int64_t npts;
  const double* exps;         // host
  const double* norms;        // host
  const double* contr;        // host
  double threshold;
  bool gga;
  int ispin = 1;              // 2: open shell, one density and one V_xc per spin
  int precision;              // PGXC_PREC_*
  int64_t max_chunk_points;   // 0: sized from free device memory
  bool keep_basis = false;    // basis values of the whole grid stay resident across builds
  bool mgga = false;          // meta-GGA: tau in the density, its term in the potential (FP64 DMMA)
  int functional = 0;         // PGXC_XC_*
};

int screen_create(ScreenPlan** out, const ScreenInput& in, const BuildArgs& a, cudaStream_t st, std::string& err);
void screen_destroy(ScreenPlan* sp);
// One build: the FP64 density matrices must be ready (a.P; for an open shell
// also Pb, the second spin's, with the same leading dimension a.ldc); E_xc /
// N_el are Kahan-added into a.acc; the packed matrix (both spins interleaved
// for an open shell) is written to ham.  With t == nullptr the build is only
// enqueued: no event records, synchronisation or host reads, so that it can be
// captured into a CUDA graph; screen_error_flag then reports a bounded wait
// of the INT8 kernels that ran out.
// Further functionals evaluated on the same density (energies only): E_xc and
// N_el of functional i are Kahan-added into acc[4 i .. 4 i + 3] ({E, cE, N,
// cN}, zeroed by the caller); with potential == false the potential
// contractions and the packing are skipped and ham is not written.
struct ScreenExtra {
  const XcConst* xc = nullptr;   // host array of n
  const int* gga = nullptr;      // host flags of n
  const int* fid = nullptr;      // host PGXC_XC_* ids of n (the meta-GGAs are evaluated by id)
  int n = 0;
  double* acc = nullptr;         // device, 4 n
  bool potential = true;
  bool tau = false;              // form tau (some functional is a meta-GGA; screen_enable_tau first)
};
int screen_run(ScreenPlan* sp, const BuildArgs& a, const double* Pb, cudaStream_t st, double* ham, ScreenTimes* t,
               std::string& err, const ScreenExtra* extra = nullptr);
int screen_error_flag(ScreenPlan* sp, cudaStream_t st, int* flag);
// The kinetic-energy density for meta-GGA energies on the density of a plan
// that does not form it in its builds: its buffer, allocated once.  Needs FP64
// gradient planes (a GGA plan of the FP64 build); PGXC_ENOTSUP otherwise.
int screen_enable_tau(ScreenPlan* sp, std::string& err);

// ---------------------------------------------------------------------------
// Sets: the screened INT8 builds of many contexts (closed shell, identity
// symmetry adaptation) run as one sequence of launches over the tiles of all
// of them: per chunk of the concatenated tile queue one basis launch per
// angular momentum, one gather, one density contraction, one functional,
// one Z quantization and one potential contraction, each walking tiles of
// many contexts (their density-matrix digits and potential matrices through
// a per-tile context table), and one packing launch for all contexts.
// Contexts are grouped by functional (a chunk holds one functional).
// ---------------------------------------------------------------------------
struct ScreenSet;
struct SetMember {
  ScreenPlan* sp;
  const BuildArgs* a;    // the context's arguments (basis tables, functional, acc)
  int functional;        // PGXC_XC_* id
  double* d_ham;         // packed matrix out (overwritten)
  double* d_exc_nel;     // {E_xc, N_el} out (overwritten)
};
// max_chunk_points: 0 -> sized from free device memory
int screen_set_create(ScreenSet** out, const std::vector<SetMember>& members, int64_t max_chunk_points,
                      cudaStream_t st, std::string& err);
void screen_set_destroy(ScreenSet* s);
// Enqueue the set's build on st (capturable: no synchronisation, events or
// host reads).  Each member's density-matrix digits (screen_mixed_prepare),
// potential accumulator (zeroed) and acc (zeroed) must be ready on st.
int screen_set_run(ScreenSet* s, cudaStream_t st, std::string& err);
int screen_set_error_flag(ScreenSet* s, cudaStream_t st, int* flag);
// A member's per-build preparation on st: its potential accumulator zeroed
// and its density matrix P (leading dimension ldc) in digit form.
int screen_set_prepare_member(ScreenPlan* sp, const double* P, int64_t ldc, cudaStream_t st);
// whether a context's plan can join a set (screened INT8, closed shell, basis not kept)
bool screen_set_eligible(const ScreenPlan* sp);
// tiles, chunks and launches of one run
void screen_set_stats(const ScreenSet* s, int64_t* ntiles, int64_t* nchunks, int64_t* launches);
// Plan statistics: tiles, total slots (padded), listed functions, sum of n_t^2.
void screen_stats(const ScreenPlan* sp, int64_t* ntiles, int64_t* nslots, int64_t* nlisted, double* sum_n2,
                  int64_t* nchunks);

}  // namespace pgxc
