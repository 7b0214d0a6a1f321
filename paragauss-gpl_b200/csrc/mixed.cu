// mixed.cu -- mixed-precision path (placeholder until the tensor-core kernels land).
#include "mixed.h"

namespace pgxc {

struct MixedState {
  int dummy;
};

int mixed_create(MixedState** out, const BuildArgs&, int64_t, bool, int, std::string& err) {
  *out = nullptr;
  err = "mixed precision is not implemented yet";
  return PGXC_ENOTSUP;
}
void mixed_destroy(MixedState* m) { delete m; }
int mixed_prepare(MixedState*, const BuildArgs&, cudaStream_t) { return 0; }
int mixed_basis(MixedState*, const BuildArgs&, int64_t, int64_t, bool, cudaStream_t) { return 0; }
int mixed_density(MixedState*, const BuildArgs&, bool, cudaStream_t) { return 0; }
int mixed_potential(MixedState*, const BuildArgs&, bool, cudaStream_t, cudaEvent_t, cudaEvent_t) { return 0; }
int mixed_pack(MixedState*, const BuildArgs&, int64_t, int, int, double*, cudaStream_t) { return 0; }

}  // namespace pgxc
