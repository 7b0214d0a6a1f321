// noalloc.cu -- Becke partition weights without any device allocation.
//
// pgxc_becke_weights copies its inputs to device memory it allocates and
// uses an allocated natoms x natoms distance matrix as scratch.  Some callers
// cannot let a library allocate: a Fortran SCF driver whose device arrays all
// come from its own OpenACC / CUDA Fortran data regions or memory pool, or a
// process that has reserved the whole device for its own allocator.  For them
// pgxc_becke_weights_noalloc takes device pointers for every input and output
// and keeps its only scratch, the atom-atom distance and reciprocal-distance
// matrices, in the fixed array below.
//
// The array is a file-scope __device__ object: it exists on every GPU that
// loads this library, from module load until process exit, and is shared by
// all calls on that GPU.  Each call overwrites the natoms*natoms entries it
// reads, so nothing needs clearing, but two calls that overlap on the GPU
// (different streams or host threads, same device) race on it.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/pgxc.h"
#include "kernels.h"

namespace {

// Largest geometry the allocation-free entry point accepts.
constexpr int kMaxAtoms = PGXC_NOALLOC_MAX_ATOMS;

// Scratch: atom-atom distances and their reciprocals, two row-major
// natoms x natoms matrices (4 MiB at the limit).
static __device__ __align__(256) double g_becke_dist[2 * kMaxAtoms * kMaxAtoms];

// Device address of g_becke_dist per device ordinal, resolved once per CUDA
// context.  In host code the name g_becke_dist is only a host-side shadow
// symbol, not a device address, so the address must come from
// cudaGetSymbolAddress on a context of that device.  The cache remembers the
// context it was resolved in: after cudaDeviceReset, or when the caller makes
// another context current on the same ordinal, the address is resolved again
// instead of reusing one that belongs to a destroyed or different context.
constexpr int kMaxDevices = 64;
struct SymbolSlot {
  void* ctx = nullptr;
  double* addr = nullptr;
};
SymbolSlot g_dist_addr[kMaxDevices];
std::mutex g_mu;

// The calling thread's current CUDA context (CUcontext as an opaque pointer),
// through the driver entry point the runtime exposes, so that the library does
// not link libcuda itself.  nullptr when the entry point is unavailable.
void* current_context() {
  using CtxGetCurrent = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrent) nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// The message is read back with pgxc_last_error(NULL).
int fail(int code, const std::string& msg) {
  pgxc::set_global_error(msg);
  return code;
}

}  // namespace

extern "C" int pgxc_becke_weights_noalloc(int32_t natoms, const double* d_coords, int64_t npts,
                                          const double* d_pts, const int32_t* d_point_atom, double* d_w_out,
                                          void* stream) {
  if (natoms <= 0 || npts < 0 || !d_coords || !d_pts || !d_point_atom || !d_w_out)
    return fail(PGXC_EINVAL, "pgxc_becke_weights_noalloc: bad arguments");
  if (natoms > kMaxAtoms)
    return fail(PGXC_EINVAL, "pgxc_becke_weights_noalloc: natoms " + std::to_string(natoms) +
                                 " exceeds the fixed scratch limit of " + std::to_string(kMaxAtoms) +
                                 " atoms; use pgxc_becke_weights");
  if (npts == 0) return PGXC_OK;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(PGXC_ENODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(PGXC_ENOTSUP, "device ordinal beyond the supported range");
  double* dist = nullptr;
  {
    // set-up on this device (the current device), once per context
    std::lock_guard<std::mutex> lock(g_mu);
    void* ctx = current_context();
    SymbolSlot& slot = g_dist_addr[dev];
    if (!slot.addr || !ctx || slot.ctx != ctx) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_becke_dist);
      if (e != cudaSuccess || !p)
        return fail(PGXC_ECUDA, std::string("cudaGetSymbolAddress(g_becke_dist): ") + cudaGetErrorString(e));
      slot.addr = static_cast<double*>(p);
      slot.ctx = ctx;
    }
    dist = slot.addr;
  }
  // d_pts is (npts, 3) column-major; the kernels write every entry they read
  // of the scratch (distance matrix) before reading it.
  e = pgxc::launch_becke(d_coords, dist, natoms, d_pts, d_pts + npts, d_pts + 2 * npts, d_point_atom, npts, d_w_out,
                         static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(PGXC_ECUDA, std::string("Becke kernels: ") + cudaGetErrorString(e));
  return PGXC_OK;
}
