// mixed.h -- the dense-layout INT8 build: FP64 basis, both contractions on
// the INT8 tensor cores (Ozaki split, exact integer accumulation), FP64
// functional and sums.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "kernels.h"

namespace pgxc {

struct MixedState;

int mixed_create(MixedState** out, const BuildArgs& a, int64_t nbas, bool gga, int precision, std::string& err);
void mixed_destroy(MixedState* m);
// functions are padded to a multiple of this in the mixed path's buffers
int64_t mixed_row_align();
// Each launcher returns the number of kernels it launched.
int mixed_prepare(MixedState* m, const BuildArgs& a, int nocc, cudaStream_t st);
// the same from a density matrix P given in device memory (ldc x ldc)
int mixed_prepare_P(MixedState* m, const double* P, int64_t ldc, cudaStream_t st);
// copies the device error flag (set by a bounded wait that ran out) to *flag and clears it
int mixed_error_flag(MixedState* m, cudaStream_t st, int* flag);
int mixed_basis(MixedState* m, const BuildArgs& a, int64_t p0, int64_t nvalid, bool gga, cudaStream_t st);
int mixed_density(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st);
// records k0 before and k1 after the potential contraction kernel
int mixed_potential(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1);
int mixed_pack(MixedState* m, const BuildArgs& a, int64_t nbas, int ispin, int spin, double* ham, cudaStream_t st);

}  // namespace pgxc
