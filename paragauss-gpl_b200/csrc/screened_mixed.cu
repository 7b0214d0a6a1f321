// screened_mixed.cu -- INT8 tensor-core stages of the screened XC build.
#include "screened_mixed.h"

namespace pgxc {

struct ScreenMixed {
  int dummy = 0;
};

int64_t screen_mixed_bytes_per_slot() { return 0; }
int64_t screen_mixed_bytes_per_tile() { return 0; }
int screen_mixed_create(ScreenMixed** out, const ScreenMixedInput&, std::string& err) {
  *out = nullptr;
  err = "screened mixed-precision build: not built yet";
  return PGXC_ENOTSUP;
}
void screen_mixed_destroy(ScreenMixed* m) { delete m; }
int screen_mixed_prepare(ScreenMixed*, const BuildArgs&, cudaStream_t) { return 0; }
int screen_mixed_basis(ScreenMixed*, const int64_t*, int64_t, int64_t, int64_t, const double*, cudaStream_t) {
  return 0;
}
int screen_mixed_density(ScreenMixed*, const int64_t*, const int*, int64_t, int64_t, int64_t, const double*,
                         const double*, const double*, const double*, double*, double*, double*, double*,
                         cudaStream_t) {
  return 0;
}
int screen_mixed_potential(ScreenMixed*, const int64_t*, const int*, const int*, int64_t, int64_t, int64_t, int64_t,
                           const double*, const double*, const double*, const double*, const double*, const double*,
                           const double*, const double*, double*, int64_t, cudaStream_t, cudaEvent_t, cudaEvent_t) {
  return 0;
}
int screen_mixed_error_flag(ScreenMixed*, cudaStream_t, int* flag) {
  *flag = 0;
  return PGXC_OK;
}

}  // namespace pgxc
