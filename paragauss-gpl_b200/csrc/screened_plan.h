// screened_plan.h -- the screening plan of one context (internal to the
// screened builds: screened.cu and the multi-context set in set_build.cu).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "basis.cuh"
#include "screened.h"
#include "screened_mixed.h"

namespace pgxc {

constexpr int kSlotAlign = 32;   // slots per tile are padded to this (INT8 K step)
constexpr int64_t kSlack = 128;  // zero rows after the last slot of a chunk
constexpr int kBasisBlocksPerSM = 16;  // blocks of the basis kernels per SM (each walks a range of items)

struct ScreenPlan {
  int64_t ntiles = 0, nslots = 0, nlisted = 0;
  double sum_n2 = 0.0;
  int max_n = 0;
  bool gga = false;
  int ispin = 1;
  int64_t nbas = 0;
  int64_t n_exps = 0, n_contr = 0, n_rng = 0;  // lengths of the context's exponent, contraction and range tables
  bool keep = false;         // basis values (and INT8 point digits) of all slots stay resident
  bool basis_ready = false;  // ... and a completed build has filled them
  // device, whole grid
  double *qx = nullptr, *qy = nullptr, *qz = nullptr, *qw = nullptr;  // Morton-ordered points [ntiles*128]
  int64_t* tso = nullptr;   // [ntiles+1] first slot of each tile
  int* slot_fn = nullptr;   // [nslots] function of each slot, -1 for padding
  int* slot_tile = nullptr; // [nslots]
  int* listed = nullptr;    // [ntiles] listed (not padding) slots of each tile
  int64_t* b_off = nullptr;  // [ntiles+1] first density B stage of each tile (INT8 path)
  BasisItem* items[kMaxL + 1] = {};
  // host copies of the partition
  std::vector<int64_t> h_tso;
  std::vector<int64_t> chunk_t0;                   // chunk c covers tiles [chunk_t0[c], chunk_t0[c+1])
  std::vector<int64_t> item_off[kMaxL + 1];        // items of chunk c: [item_off[L][c], item_off[L][c+1])
  std::vector<int64_t> tile_item[kMaxL + 1];       // items before tile t, per L ([ntiles + 1])
  int64_t chunk_slots = 0, chunk_tiles = 0;        // buffer capacities
  // device, per chunk
  double *phi = nullptr, *gx = nullptr, *gy = nullptr, *gz = nullptr, *Z = nullptr;
  // INT8 build (not a meta-GGA): grad phi in 32-bit planes instead of gx/gy/gz
  bool gf32 = false;
  float *fx = nullptr, *fy = nullptr, *fz = nullptr;
  double* pt = nullptr;      // 8 point arrays of chunk_tiles*128 per spin
  bool mgga = false;
  int functional = 0;        // PGXC_XC_* (the meta-GGA step selects its functional by id)
  double* tq = nullptr;      // meta-GGA: 4 point arrays per spin (2 tau_x, 2 tau_y, 2 tau_z, C)
  double* partial = nullptr;
  double* V = nullptr;       // [ispin][nbas][nbas]
  unsigned long long* pmax = nullptr;  // [chunk_tiles*128] largest |phi| per point (INT8 path)
  ScreenMixed* mixed = nullptr;
  cudaEvent_t ev[12] = {};
  int nsm = 148;
  std::vector<void*> allocs;
};


}  // namespace pgxc
