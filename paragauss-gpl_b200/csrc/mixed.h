// mixed.h -- the mixed-precision (FP32 basis, split BF16x3 / TF32x3 tensor-core
// contractions, FP64 functional and sums) path of the XC build.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "kernels.h"

namespace pgxc {

struct MixedState;

int mixed_create(MixedState** out, const BuildArgs& a, int64_t nbas, bool gga, int precision, std::string& err);
void mixed_destroy(MixedState* m);
// Each launcher returns the number of kernels it launched.
int mixed_prepare(MixedState* m, const BuildArgs& a, cudaStream_t st);
int mixed_basis(MixedState* m, const BuildArgs& a, int64_t p0, int64_t nvalid, bool gga, cudaStream_t st);
int mixed_density(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st);
// records k0 before and k1 after the potential contraction kernel
int mixed_potential(MixedState* m, const BuildArgs& a, bool gga, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1);
int mixed_pack(MixedState* m, const BuildArgs& a, int64_t nbas, int ispin, int spin, double* ham, cudaStream_t st);

}  // namespace pgxc
