// pgxc_api.cu -- the C ABI of libpgxc (include/pgxc.h).
//
// One context per geometry (pgxc_create, where ParaGauss runs xc_setup),
// one pgxc_build per SCF cycle (in place of calc_xcks / calc_xcks_nl).
// Everything is computed on the device; a missing or unusable CUDA device is
// an error (PGXC_ENODEV), never a CPU fallback.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gradient.h"
#include "grid.h"
#include "kernels.h"
#include "mixed.h"
#include "pgxc_common.cuh"
#include "screened.h"
#include "symmetry.h"

using namespace pgxc;

// Symmetry adaptation of a context (pgxc_set_symmetry): the device tables and
// the host sizes a symmetric build needs.
struct SymPlan {
  SymDev dev;
  std::vector<int> dims, partners, ipbase;
  std::vector<int64_t> pkofs;
  int nip = 0, max_dim = 0;
  int64_t len = 0;                 // sum_i dims_i (dims_i + 1) / 2
  double* d_ham = nullptr;         // ispin * len packed symmetric matrix
  double* d_Csa = nullptr;         // the irreps' orbitals of one build
  int64_t csa_cap = 0;
  int64_t* d_cofs = nullptr;       // [ispin * n_irrep]
  int* d_nocc = nullptr;           // [n_irrep]
  int64_t* d_col0 = nullptr;       // [nip]
  // pseudo-2D irreps (pgxc_set_pseudo2d)
  Pseudo2dPair* d_p2 = nullptr;
  int64_t* d_p2first = nullptr;
  int64_t p2_pairs = 0, p2_quads = 0;
};

struct pgxc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  cudaEvent_t kev[4] = {};
  std::string err;
  pgxc_options opt;
  int natm = 0;
  int64_t nbas = 0, npts = 0;
  int lmax = 0;
  BuildArgs a;
  std::vector<void*> allocs;
  // host copies needed later
  std::vector<DevShell> shells;
  // device buffers not in BuildArgs
  double* d_ham = nullptr;
  double* d_dist = nullptr;
  // open shell: the second spin's orbitals, occupations and density matrix
  double* C2 = nullptr;
  double* occ2 = nullptr;
  double* P2 = nullptr;
  int nocc_cap = 0;
  int64_t chunk = 0;
  double* h_ham = nullptr;      // pinned staging for the packed matrix
  double* h_acc = nullptr;      // pinned {E, cE, N, cN}
  MixedState* mixed = nullptr;  // tensor-core mixed-precision path (dense)
  ScreenPlan* screen = nullptr; // screened (tile-sparse) build, when screen_threshold >= 0
  SymPlan* sym = nullptr;       // symmetry adaptation, when set
  double* d_eacc = nullptr;     // {E, cE, N, cN} per functional of pgxc_xc_energies
  void* grad_scr = nullptr;     // scratch of pgxc_xc_gradient, kept across calls (grows only)
  size_t grad_scr_bytes = 0;
  int eacc_cap = 0;
  int* d_owner = nullptr;       // host atom of each point (raw-weight grids)
  double* d_wraw = nullptr;     // the raw weights of those grids
};

namespace {

thread_local std::string g_err;

int set_err(pgxc_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  g_err = msg;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                     \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return set_err(ctx, e_ == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA,           \
                     std::string(#call " failed: ") + cudaGetErrorString(e_));                  \
  } while (0)

template <typename T>
int dalloc(pgxc_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess)
    return set_err(c, PGXC_ENOMEM, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) +
                                       " bytes failed: " + cudaGetErrorString(e));
  c->allocs.push_back(q);
  *p = (T*)q;
  return PGXC_OK;
}

int check_device(pgxc_ctx* c, int want) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return set_err(c, PGXC_ENODEV, "no CUDA device available");
  int dev = want;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) return set_err(c, PGXC_ENODEV, "cudaGetDevice failed");
  }
  if (dev >= n) return set_err(c, PGXC_EINVAL, "device ordinal out of range");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return set_err(c, PGXC_ENODEV, "device query failed");
  if (prop.major != 10) return set_err(c, PGXC_ENODEV, "libpgxc is built for sm_100a (B200) only");
  if (c) c->device = dev;
  return PGXC_OK;
}

bool all_finite(const double* p, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// A device copy of a host vector (a context allocation).
template <typename T>
int upload_vec(pgxc_ctx* c, const std::vector<T>& v, T** d) {
  int st = dalloc(c, d, v.size());
  if (st) return st;
  if (!v.empty()) CUDA_TRY(c, cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return PGXC_OK;
}

}  // namespace

void pgxc::set_global_error(const std::string& msg) { g_err = msg; }

extern "C" {

void pgxc_default_options(pgxc_options* o) {
  if (!o) return;
  o->functional = PGXC_XC_VWN;
  o->ispin = 1;
  o->precision = PGXC_PREC_FP64;
  o->batch_points = 128;
  o->screen_threshold = 0.0;
  o->device = -1;
  o->keep_orbitals = 0;
  o->max_chunk_points = 0;
}

const char* pgxc_last_error(const pgxc_ctx* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

const char* pgxc_strerror(int s) {
  switch (s) {
    case PGXC_OK: return "ok";
    case PGXC_EINVAL: return "invalid argument";
    case PGXC_ENOTSUP: return "not supported";
    case PGXC_ENOMEM: return "out of device memory";
    case PGXC_ECUDA: return "CUDA error";
    case PGXC_ETIMEOUT: return "device wait timed out";
    case PGXC_ENONFINITE: return "non-finite value";
    case PGXC_ENODEV: return "no usable CUDA device";
    default: return "unknown status";
  }
}

void pgxc_destroy(pgxc_ctx* c) {
  if (!c) return;
  if (c->device >= 0) cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->mixed) mixed_destroy(c->mixed);
  if (c->screen) screen_destroy(c->screen);
  delete c->sym;
  for (void* p : c->allocs) cudaFree(p);
  if (c->grad_scr) cudaFree(c->grad_scr);
  if (c->h_ham) cudaFreeHost(c->h_ham);
  if (c->h_acc) cudaFreeHost(c->h_acc);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->kev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int pgxc_screen_stats(const pgxc_ctx* c, int64_t* ntiles, int64_t* nslots, int64_t* nlisted, double* sum_n2) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  if (!c->screen) return set_err(const_cast<pgxc_ctx*>(c), PGXC_EINVAL, "context has no screening plan");
  screen_stats(c->screen, ntiles, nslots, nlisted, sum_n2, nullptr);
  return PGXC_OK;
}

int pgxc_nbas(const pgxc_ctx* c, int32_t* nbas) {
  if (!c || !nbas) return PGXC_EINVAL;
  *nbas = (int32_t)c->nbas;
  return PGXC_OK;
}

static int validate_basis(pgxc_ctx* c, const pgxc_geometry* geo, const pgxc_basis* b, std::vector<DevShell>& out,
                          int64_t& nbas, int& lmax, int64_t& nexp_tot, int64_t& ncon_tot) {
  if (!geo || !b || geo->natoms <= 0 || !geo->coords || b->nshells <= 0)
    return set_err(c, PGXC_EINVAL, "empty geometry or basis");
  if (!b->shell_atom || !b->shell_l || !b->shell_nexp || !b->shell_nunc || !b->shell_ncontr || !b->exponents ||
      !b->norms || !b->contractions)
    return set_err(c, PGXC_EINVAL, "basis arrays must not be NULL");
  int last_atom = -1, last_l = -1;
  nbas = 0;
  lmax = 0;
  nexp_tot = 0;
  ncon_tot = 0;
  for (int s = 0; s < b->nshells; ++s) {
    DevShell S{};
    S.atom = b->shell_atom[s];
    S.l = b->shell_l[s];
    S.nexp = b->shell_nexp[s];
    S.nunc = b->shell_nunc[s];
    S.ncontr = b->shell_ncontr[s];
    if (S.atom < 0 || S.atom >= geo->natoms) return set_err(c, PGXC_EINVAL, "shell atom index out of range");
    if (S.l < 0) return set_err(c, PGXC_EINVAL, "negative l");
    if (S.l > kMaxL) return set_err(c, PGXC_ENOTSUP, "l > 3 is not supported");
    if (S.nexp <= 0 || S.nunc < 0 || S.ncontr < 0 || S.nunc > S.nexp)
      return set_err(c, PGXC_EINVAL, "bad shell exponent/contraction counts");
    if (S.nunc + S.ncontr > 64) return set_err(c, PGXC_ENOTSUP, "more than 64 radial functions in one shell");
    if (S.atom < last_atom || (S.atom == last_atom && S.l <= last_l))
      return set_err(c, PGXC_EINVAL, "shells must be ordered by atom, then l (orbitalprojection order)");
    last_atom = S.atom;
    last_l = S.l;
    S.nrad = S.nunc + S.ncontr;
    S.exp_off = (int)nexp_tot;
    S.con_off = (int)ncon_tot;
    S.f0 = (int)nbas;
    double mn = 1e300;
    for (int e = 0; e < S.nexp; ++e) {
      const double a = b->exponents[nexp_tot + e];
      if (!(a > 0.0) || !std::isfinite(a)) return set_err(c, PGXC_EINVAL, "exponents must be positive and finite");
      mn = std::min(mn, a);
    }
    S.min_exp = mn;
    nexp_tot += S.nexp;
    ncon_tot += (int64_t)S.nexp * S.ncontr;
    nbas += (int64_t)(2 * S.l + 1) * S.nrad;
    lmax = std::max(lmax, S.l);
    out.push_back(S);
  }
  if (!all_finite(b->norms, nexp_tot) || !all_finite(b->contractions, ncon_tot) ||
      !all_finite(geo->coords, 3 * (int64_t)geo->natoms))
    return set_err(c, PGXC_ENONFINITE, "non-finite basis or geometry input");
  if (nbas == 0) return set_err(c, PGXC_EINVAL, "basis has no functions");
  return PGXC_OK;
}

namespace {

// Grid of a spec: shells kept per atom (r < 40 bohr) and the first point of each atom.
int spec_layout(pgxc_ctx* c, const pgxc_geometry* geo, const pgxc_grid_spec* spec, std::vector<int64_t>& off,
                std::vector<double>& ang) {
  if (!geo || geo->natoms <= 0 || !geo->coords) return set_err(c, PGXC_EINVAL, "bad geometry");
  if (!spec || !spec->nrad || !spec->radius) return set_err(c, PGXC_EINVAL, "grid spec needs nrad and radius");
  if (lebedev_rule(spec->nang, ang) != 0)
    return set_err(c, PGXC_EINVAL, "no Lebedev-McLaren rule with " + std::to_string(spec->nang) +
                                       " points (6, 8, 12, 14, 26, 38, 50, 78, 86, 110, 146, 194, 302)");
  off.assign((size_t)geo->natoms + 1, 0);
  for (int a = 0; a < geo->natoms; ++a) {
    if (spec->nrad[a] <= 0 || !(spec->radius[a] > 0.0) || !std::isfinite(spec->radius[a]))
      return set_err(c, PGXC_EINVAL, "grid spec: nrad and radius must be positive");
    off[(size_t)a + 1] = off[(size_t)a] + radial_shells(spec->nrad[a], spec->radius[a]) * spec->nang;
  }
  return PGXC_OK;
}

// The spec's grid into device arrays gx, gy, gz, gw (SoA, n points) and owner.
int spec_generate(pgxc_ctx* c, const pgxc_geometry* geo, const pgxc_grid_spec* spec, const std::vector<int64_t>& off,
                  const std::vector<double>& ang, double* gx, double* gy, double* gz, double* gw, int* owner,
                  cudaStream_t st) {
  const int natm = geo->natoms;
  const int64_t n = off.back();
  double *datoms = nullptr, *drc = nullptr, *dang = nullptr;
  int64_t* doff = nullptr;
  int* dnr = nullptr;
  cudaError_t e = cudaMalloc(&datoms, sizeof(double) * 3 * natm);
  if (e == cudaSuccess) e = cudaMalloc(&drc, sizeof(double) * natm);
  if (e == cudaSuccess) e = cudaMalloc(&dang, sizeof(double) * ang.size());
  if (e == cudaSuccess) e = cudaMalloc(&doff, sizeof(int64_t) * off.size());
  if (e == cudaSuccess) e = cudaMalloc(&dnr, sizeof(int) * natm);
  const bool oom = e == cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaMemcpy(datoms, geo->coords, sizeof(double) * 3 * natm, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(drc, spec->radius, sizeof(double) * natm, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dang, ang.data(), sizeof(double) * ang.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(doff, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dnr, spec->nrad, sizeof(int) * natm, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = launch_atomic_grid(natm, datoms, doff, drc, dnr, dang, spec->nang, n, gx, gy, gz, gw, owner, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(datoms);
  cudaFree(drc);
  cudaFree(dang);
  cudaFree(doff);
  cudaFree(dnr);
  if (e != cudaSuccess)
    return set_err(c, oom ? PGXC_ENOMEM : PGXC_ECUDA, std::string("atomic grid: ") + cudaGetErrorString(e));
  return PGXC_OK;
}

// pgxc_create with either a host grid or a grid spec (exactly one non-NULL)
int create_impl(const pgxc_geometry* geo, const pgxc_basis* bas, const pgxc_grid* grid, const pgxc_grid_spec* spec,
                const pgxc_options* opt, pgxc_ctx** out) {
  if (!out) return set_err(nullptr, PGXC_EINVAL, "out is NULL");
  *out = nullptr;
  pgxc_ctx* c = new (std::nothrow) pgxc_ctx();
  if (!c) return set_err(nullptr, PGXC_ENOMEM, "host allocation failed");
  pgxc_options o;
  pgxc_default_options(&o);
  if (opt) o = *opt;
  if (o.batch_points <= 0) o.batch_points = 128;
  c->opt = o;
  auto fail = [&](int st) {
    g_err = c->err;
    pgxc_destroy(c);
    return st;
  };
  if (o.functional < PGXC_XC_VWN || o.functional > PGXC_XC_LAST)
    return fail(set_err(c, PGXC_EINVAL, "unknown functional id"));
  if (o.ispin != 1 && o.ispin != 2) return fail(set_err(c, PGXC_EINVAL, "ispin must be 1 or 2"));
  if (o.ispin == 2 && !(o.screen_threshold >= 0.0))
    return fail(set_err(c, PGXC_ENOTSUP, "open-shell (ispin=2) builds need the screened layout (screen_threshold >= 0)"));
  if (PGXC_XC_IS_MGGA(o.functional) && !(o.screen_threshold >= 0.0))
    return fail(set_err(c, PGXC_ENOTSUP, "meta-GGA builds need the screened layout (screen_threshold >= 0)"));
  if (o.precision != PGXC_PREC_FP64 && o.precision != PGXC_PREC_MIXED_INT8)
    return fail(set_err(c, PGXC_EINVAL, "unknown precision mode"));
  std::vector<int64_t> spec_off;
  std::vector<double> spec_ang;
  if (spec) {
    int sst = spec_layout(c, geo, spec, spec_off, spec_ang);
    if (sst) return fail(sst);
    if (spec_off.back() <= 0) return fail(set_err(c, PGXC_EINVAL, "empty grid"));
  } else {
    if (!grid || grid->npts <= 0 || !grid->grdpts) return fail(set_err(c, PGXC_EINVAL, "empty grid"));
    if (grid->weights_are_raw && !grid->point_atom)
      return fail(set_err(c, PGXC_EINVAL, "raw weights need point_atom"));
  }
  int64_t nexp_tot, ncon_tot;
  int st = validate_basis(c, geo, bas, c->shells, c->nbas, c->lmax, nexp_tot, ncon_tot);
  if (st) return fail(st);
  if (!spec) {
    if (!all_finite(grid->grdpts, 4 * grid->npts)) return fail(set_err(c, PGXC_ENONFINITE, "non-finite grid input"));
    if (grid->weights_are_raw)
      for (int64_t i = 0; i < grid->npts; ++i)
        if (grid->point_atom[i] < 0 || grid->point_atom[i] >= geo->natoms)
          return fail(set_err(c, PGXC_EINVAL, "point_atom out of range"));
  }
  const bool raw_weights = spec || grid->weights_are_raw;
  st = check_device(c, o.device);
  if (st) return fail(st);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(set_err(c, PGXC_ECUDA, "cudaSetDevice failed"));
  CUDA_TRY(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (auto& e : c->ev) CUDA_TRY(c, cudaEventCreate(&e));
  for (auto& e : c->kev) CUDA_TRY(c, cudaEventCreate(&e));
  c->natm = geo->natoms;
  c->npts = spec ? spec_off.back() : grid->npts;
  BuildArgs& a = c->a;
  a.nshells = (int)c->shells.size();
  a.xc = make_xc_const(o.functional);
  // symmetry adaptation table
  std::memset(&a.sa, 0, sizeof(a.sa));
  a.sa.identity = 1;
  if (bas->sa_coef) {
    if (bas->sa_lmax < c->lmax) return fail(set_err(c, PGXC_EINVAL, "sa_coef must cover every l of the basis"));
    int64_t off = 0;
    for (int l = 0; l <= std::min(bas->sa_lmax, kMaxL); ++l) {
      const int n = 2 * l + 1;
      for (int i = 0; i < n; ++i)
        for (int m = 0; m < n; ++m) {
          const double v = bas->sa_coef[off + i * n + m];
          a.sa.c[l][i][m] = v;
          if (v != (i == m ? 1.0 : 0.0)) a.sa.identity = 0;
        }
      off += n * n;
    }
  }
  // basis and geometry
  DevShell* dsh;
  double *datoms, *dexps, *dnorms, *dcontr;
  if ((st = dalloc(c, &dsh, c->shells.size())) || (st = dalloc(c, &datoms, 3 * (size_t)c->natm)) ||
      (st = dalloc(c, &dexps, nexp_tot)) || (st = dalloc(c, &dnorms, nexp_tot)) ||
      (st = dalloc(c, &dcontr, std::max<int64_t>(ncon_tot, 1))))
    return fail(st);
  CUDA_TRY(c, cudaMemcpy(dsh, c->shells.data(), c->shells.size() * sizeof(DevShell), cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(datoms, geo->coords, 3 * sizeof(double) * c->natm, cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(dexps, bas->exponents, sizeof(double) * nexp_tot, cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(dnorms, bas->norms, sizeof(double) * nexp_tot, cudaMemcpyHostToDevice));
  if (ncon_tot) CUDA_TRY(c, cudaMemcpy(dcontr, bas->contractions, sizeof(double) * ncon_tot, cudaMemcpyHostToDevice));
  a.shells = dsh;
  {
    // contraction ranges: a shell is segmented when it has no bare primitives
    // and every contraction's nonzero coefficients form its own contiguous,
    // disjoint range of primitives (each primitive then feeds one function)
    std::vector<int2> rng;
    for (DevShell& S : c->shells) {
      S.seg = 0;
      S.rad_off = (int)rng.size();
      if (S.nunc != 0 || S.ncontr == 0) continue;
      std::vector<int2> r((size_t)S.ncontr);
      bool seg = true;
      std::vector<int> owner((size_t)S.nexp, -1);
      for (int j = 0; j < S.ncontr && seg; ++j) {
        int lo = -1, hi = -1;
        for (int e = 0; e < S.nexp; ++e)
          if (bas->contractions[S.con_off + e + (int64_t)S.nexp * j] != 0.0) {
            if (lo < 0) lo = e;
            hi = e + 1;
          }
        if (lo < 0) lo = hi = 0;
        for (int e = lo; e < hi && seg; ++e) {
          if (owner[(size_t)e] >= 0) seg = false;
          owner[(size_t)e] = j;
        }
        r[(size_t)j] = make_int2(lo, hi);
      }
      if (!seg) continue;
      S.seg = 1;
      rng.insert(rng.end(), r.begin(), r.end());
    }
    int2* drng = nullptr;
    if ((st = dalloc(c, &drng, std::max<size_t>(rng.size(), 1)))) return fail(st);
    if (!rng.empty()) CUDA_TRY(c, cudaMemcpy(drng, rng.data(), rng.size() * sizeof(int2), cudaMemcpyHostToDevice));
    a.rng = drng;
    CUDA_TRY(c, cudaMemcpy(dsh, c->shells.data(), c->shells.size() * sizeof(DevShell), cudaMemcpyHostToDevice));
  }
  {
    std::vector<int> ids[kMaxL + 1];
    for (int i = 0; i < (int)c->shells.size(); ++i) ids[c->shells[i].l].push_back(i);
    for (int l = 0; l <= kMaxL; ++l) {
      a.nshl[l] = (int)ids[l].size();
      int* d = nullptr;
      if ((st = dalloc(c, &d, std::max<size_t>(ids[l].size(), 1)))) return fail(st);
      if (!ids[l].empty()) CUDA_TRY(c, cudaMemcpy(d, ids[l].data(), ids[l].size() * sizeof(int), cudaMemcpyHostToDevice));
      a.shl[l] = d;
    }
  }
  a.atoms = datoms;
  a.exps = dexps;
  a.norms = dnorms;
  a.contr = dcontr;
  // grid, SoA
  const int64_t n = c->npts;
  double* dgrid;
  if ((st = dalloc(c, &dgrid, 4 * (size_t)n))) return fail(st);
  if (!spec) CUDA_TRY(c, cudaMemcpy(dgrid, grid->grdpts, 4 * sizeof(double) * n, cudaMemcpyHostToDevice));
  a.px = dgrid;
  a.py = dgrid + n;
  a.pz = dgrid + 2 * n;
  a.w = dgrid + 3 * n;
  if (raw_weights) {
    // w <- w_raw * Becke partition weight of the host atom (mkgrid :3135-3137)
    int* downer;
    double* dbecke;
    if ((st = dalloc(c, &downer, n)) || (st = dalloc(c, &dbecke, n)) ||
        (st = dalloc(c, &c->d_dist, 2 * (size_t)c->natm * c->natm)))
      return fail(st);
    if (spec) {
      // the grid itself is built on the device (grid_main_calc)
      if ((st = spec_generate(c, geo, spec, spec_off, spec_ang, dgrid, dgrid + n, dgrid + 2 * n, dgrid + 3 * n, downer,
                              c->stream)))
        return fail(st);
    } else {
      CUDA_TRY(c, cudaMemcpy(downer, grid->point_atom, sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    // the raw weights and hosts stay for the nuclear gradient (pgxc_xc_gradient)
    if ((st = dalloc(c, &c->d_wraw, n))) return fail(st);
    CUDA_TRY(c, cudaMemcpy(c->d_wraw, dgrid + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    c->d_owner = downer;
    CUDA_TRY(c, launch_becke(datoms, c->d_dist, c->natm, a.px, a.py, a.pz, downer, n, dbecke, c->stream));
    launch_scale_inplace(dgrid + 3 * n, dbecke, n, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  a.ldc = round_up(c->nbas, kTile);
  const bool gga = PGXC_XC_IS_GGA(o.functional);
  if (o.screen_threshold >= 0.0) {
    // screened build: per-tile significant-function lists; only P, the
    // accumulators and the packed matrix are shared with the dense layout
    if ((st = dalloc(c, &a.acc, 4)) || (st = dalloc(c, &a.P, (size_t)a.ldc * a.ldc))) return fail(st);
    if (o.ispin == 2 && (st = dalloc(c, &c->P2, (size_t)a.ldc * a.ldc))) return fail(st);
    if ((st = dalloc(c, &c->d_ham, (size_t)o.ispin * c->nbas * (c->nbas + 1) / 2))) return fail(st);
    CUDA_TRY(c, cudaMallocHost(&c->h_ham, sizeof(double) * o.ispin * c->nbas * (c->nbas + 1) / 2));
    CUDA_TRY(c, cudaMallocHost(&c->h_acc, sizeof(double) * 4));
    ScreenInput in;
    in.shells = &c->shells;
    in.atoms = geo->coords;
    in.natm = c->natm;
    in.nbas = c->nbas;
    in.npts = n;
    in.exps = bas->exponents;
    in.norms = bas->norms;
    in.contr = bas->contractions;
    in.threshold = o.screen_threshold;
    in.gga = gga;
    in.ispin = o.ispin;
    in.precision = o.precision;
    in.keep_basis = o.keep_orbitals != 0;
    in.mgga = PGXC_XC_IS_MGGA(o.functional);
    in.functional = o.functional;
    in.max_chunk_points = o.max_chunk_points;
    std::string e;
    st = screen_create(&c->screen, in, a, c->stream, e);
    if (st) return fail(set_err(c, st, e));
    *out = c;
    return PGXC_OK;
  }
  // potential tiles of the FP64 path and their split over points
  a.nt = (int)(a.ldc / kTile);
  a.ntiles = a.nt * (a.nt + 1) / 2;
  const int ns64 = (int)std::min<int64_t>(8, std::max<int64_t>(1, (2 * 148 + a.ntiles - 1) / a.ntiles));
  // chunk sizing: balanced chunks of at most max_chunk points, each a
  // multiple of 128 * ns64 (CTA rows of both paths, 16-point K slabs per split)
  size_t freeb = 0, totb = 0;
  CUDA_TRY(c, cudaMemGetInfo(&freeb, &totb));
  const int64_t arrays = gga ? 5 : 2;
  // FP64 path: phi (+ 3 gradients) and Z in FP64; mixed path: the same in FP64
  // plus three 5-byte operand tile sets
  const int64_t row_bytes = o.precision == PGXC_PREC_FP64 ? a.ldc * 8 : round_up(c->nbas, mixed_row_align()) * 8;
  const int64_t per_pt = row_bytes * arrays + (o.precision == PGXC_PREC_FP64 ? 0 : round_up(c->nbas, mixed_row_align()) * 15) + 8 * 10;
  const int64_t align = 128LL * ns64;
  int64_t max_chunk = (int64_t)(0.30 * (double)freeb) / per_pt;
  max_chunk = std::min<int64_t>(max_chunk, 1 << 19);
  if (o.max_chunk_points > 0) max_chunk = std::min<int64_t>(max_chunk, o.max_chunk_points);
  max_chunk = std::max<int64_t>(align, max_chunk / align * align);
  const int64_t nchunks = (n + max_chunk - 1) / max_chunk;
  const int64_t chunk = round_up((n + nchunks - 1) / nchunks, align);
  c->chunk = chunk;
  a.ldp = chunk;
  if (o.precision == PGXC_PREC_FP64) {
    if ((st = dalloc(c, &a.phi, (size_t)a.ldc * chunk)) || (st = dalloc(c, &a.Z, (size_t)a.ldc * chunk)))
      return fail(st);
    if (gga && ((st = dalloc(c, &a.gx, (size_t)a.ldc * chunk)) || (st = dalloc(c, &a.gy, (size_t)a.ldc * chunk)) ||
                (st = dalloc(c, &a.gz, (size_t)a.ldc * chunk))))
      return fail(st);
    // rows nbas..ldc-1 stay zero for ever (the basis kernel never writes them)
    CUDA_TRY(c, cudaMemset(a.phi, 0, sizeof(double) * a.ldc * chunk));
    if (gga) {
      CUDA_TRY(c, cudaMemset(a.gx, 0, sizeof(double) * a.ldc * chunk));
      CUDA_TRY(c, cudaMemset(a.gy, 0, sizeof(double) * a.ldc * chunk));
      CUDA_TRY(c, cudaMemset(a.gz, 0, sizeof(double) * a.ldc * chunk));
    }
  }
  double* pp;
  if ((st = dalloc(c, &pp, 8 * (size_t)chunk))) return fail(st);
  a.rho = pp; a.grx = pp + chunk; a.gry = pp + 2 * chunk; a.grz = pp + 3 * chunk;
  a.A = pp + 4 * chunk; a.Bx = pp + 5 * chunk; a.By = pp + 6 * chunk; a.Bz = pp + 7 * chunk;
  if ((st = dalloc(c, &a.partial, 2 * (size_t)((chunk + 255) / 256) + 2)) || (st = dalloc(c, &a.acc, 4)))
    return fail(st);
  if ((st = dalloc(c, &a.P, (size_t)a.ldc * a.ldc))) return fail(st);
  // potential tiles: upper triangle of 64x64 tiles, split over points
  {
    std::vector<int2> tl;
    std::vector<int> tof((size_t)a.nt * a.nt, -1);
    for (int I = 0; I < a.nt; ++I)
      for (int J = I; J < a.nt; ++J) {
        tof[(size_t)I * a.nt + J] = (int)tl.size();
        tl.push_back(make_int2(I, J));
      }
    int2* dtl;
    int* dtof;
    if ((st = dalloc(c, &dtl, tl.size())) || (st = dalloc(c, &dtof, tof.size()))) return fail(st);
    CUDA_TRY(c, cudaMemcpy(dtl, tl.data(), tl.size() * sizeof(int2), cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(dtof, tof.data(), tof.size() * sizeof(int), cudaMemcpyHostToDevice));
    a.tiles = dtl;
    a.tile_of = dtof;
  }
  a.nsplit = ns64;
  a.kspan = chunk / ns64;
  if ((st = dalloc(c, &a.vpart, (size_t)a.nsplit * a.ntiles * kTile * kTile))) return fail(st);
  if ((st = dalloc(c, &c->d_ham, (size_t)o.ispin * c->nbas * (c->nbas + 1) / 2))) return fail(st);
  CUDA_TRY(c, cudaMallocHost(&c->h_ham, sizeof(double) * o.ispin * c->nbas * (c->nbas + 1) / 2));
  CUDA_TRY(c, cudaMallocHost(&c->h_acc, sizeof(double) * 4));
  if (o.precision != PGXC_PREC_FP64) {
    st = mixed_create(&c->mixed, a, c->nbas, gga, o.precision, c->err);
    if (st) return fail(st);
  }
  *out = c;
  return PGXC_OK;
}

}  // namespace

int pgxc_create(const pgxc_geometry* geo, const pgxc_basis* bas, const pgxc_grid* grid, const pgxc_options* opt,
                pgxc_ctx** out) {
  return create_impl(geo, bas, grid, nullptr, opt, out);
}

int pgxc_create_on_grid(const pgxc_geometry* geo, const pgxc_basis* bas, const pgxc_grid_spec* spec,
                        const pgxc_options* opt, pgxc_ctx** out) {
  if (!spec) return set_err(nullptr, PGXC_EINVAL, "spec is NULL");
  return create_impl(geo, bas, nullptr, spec, opt, out);
}

int pgxc_atomic_grid_size(const pgxc_geometry* geo, const pgxc_grid_spec* spec, int64_t* npts) {
  if (!npts) return set_err(nullptr, PGXC_EINVAL, "npts is NULL");
  std::vector<int64_t> off;
  std::vector<double> ang;
  int st = spec_layout(nullptr, geo, spec, off, ang);
  if (st) return st;
  *npts = off.back();
  return PGXC_OK;
}

int pgxc_atomic_grid(const pgxc_geometry* geo, const pgxc_grid_spec* spec, int64_t npts, double* d_grdpts,
                     int32_t* d_point_atom, void* stream) {
  std::vector<int64_t> off;
  std::vector<double> ang;
  int st = spec_layout(nullptr, geo, spec, off, ang);
  if (st) return st;
  if (npts != off.back())
    return set_err(nullptr, PGXC_EINVAL, "npts must be " + std::to_string(off.back()) + " (pgxc_atomic_grid_size)");
  if (!d_grdpts || !d_point_atom) return set_err(nullptr, PGXC_EINVAL, "NULL output");
  if ((st = check_device(nullptr, -1))) return st;
  return spec_generate(nullptr, geo, spec, off, ang, d_grdpts, d_grdpts + npts, d_grdpts + 2 * npts,
                       d_grdpts + 3 * npts, d_point_atom, static_cast<cudaStream_t>(stream));
}


// Ensure C / occ buffers for nocc orbitals.
static int ensure_occ(pgxc_ctx* c, int nocc) {
  const int kpad = (int)round_up(std::max(nocc, 1), 16);
  if (kpad <= c->nocc_cap) return PGXC_OK;
  BuildArgs& a = c->a;
  double *C, *Cocc, *occ;
  int st;
  if ((st = dalloc(c, &C, (size_t)kpad * a.ldc)) || (st = dalloc(c, &Cocc, (size_t)kpad * a.ldc)) ||
      (st = dalloc(c, &occ, kpad)))
    return st;
  if (c->opt.ispin == 2 && ((st = dalloc(c, &c->C2, (size_t)kpad * a.ldc)) || (st = dalloc(c, &c->occ2, kpad))))
    return st;
  a.C = C;
  a.Cocc = Cocc;
  a.occ = occ;
  c->nocc_cap = kpad;
  return PGXC_OK;
}

// Copy the orbitals C (nbas x nocc per spin, spin blocks of nbas*nocc) and the
// occupations (nocc per spin) into the padded device buffers: spin a into
// a.C / a.occ, spin b (open shell) into C2 / occ2.  Padding rows and columns are zero.
static int upload_orbitals(pgxc_ctx* c, const double* C, const double* occ, int32_t nbas, int32_t nocc, int64_t kpad,
                           cudaMemcpyKind kind) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  for (int sp = 0; sp < c->opt.ispin; ++sp) {
    double* dC = sp ? c->C2 : a.C;
    double* docc = sp ? c->occ2 : (double*)a.occ;
    CUDA_TRY(c, cudaMemsetAsync(dC, 0, sizeof(double) * kpad * a.ldc, s));
    CUDA_TRY(c, cudaMemsetAsync(docc, 0, sizeof(double) * kpad, s));
    if (nocc > 0) {
      CUDA_TRY(c, cudaMemcpy2DAsync(dC, sizeof(double) * a.ldc, C + (size_t)sp * nbas * nocc, sizeof(double) * nbas,
                                    sizeof(double) * nbas, nocc, kind, s));
      CUDA_TRY(c, cudaMemcpyAsync(docc, occ + (size_t)sp * nocc, sizeof(double) * nocc, kind, s));
    }
  }
  return PGXC_OK;
}

// The device part of a build; C / occ already in a.C / a.occ (padded).
// p_given: the density matrices are already in a.P (and P2), written by the caller's P.
static int run_build(pgxc_ctx* c, int nocc, pgxc_timings* tm, bool p_given = false) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  const bool gga = PGXC_XC_IS_GGA(c->opt.functional);
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  if (c->screen) {
    CUDA_TRY(c, cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), s));
    CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
    if (!p_given) launch_pmat_f64(a, kpad, s);
    if (c->opt.ispin == 2 && !p_given) {
      BuildArgs b = a;  // second spin: its orbitals and occupations into P2 (Cocc is scratch)
      b.C = c->C2;
      b.occ = c->occ2;
      b.P = c->P2;
      launch_pmat_f64(b, kpad, s);
    }
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaEventRecord(c->ev[2], s));
    ScreenTimes T;
    std::string e;
    const int st = screen_run(c->screen, a, c->P2, s, c->d_ham, &T, e);
    if (st) return set_err(c, st, e);
    float ms = 0;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]));
    if (tm) {
      tm->basis_ms = T.basis;
      tm->density_ms = T.density + ms;
      tm->functional_ms = T.functional;
      tm->potential_ms = T.potential;
      tm->xgemm_ms = T.x;
      tm->vgemm_ms = T.v;
      tm->kernel_launches = T.launches + (p_given ? 0 : 2 * c->opt.ispin);
    }
    return PGXC_OK;
  }
  float t_basis = 0, t_dens = 0, t_func = 0, t_pot = 0, t_x = 0, t_v = 0;
  int64_t launches = 0;
  CUDA_TRY(c, cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), s));
  CUDA_TRY(c, cudaMemsetAsync(a.vpart, 0, sizeof(double) * a.nsplit * a.ntiles * kTile * kTile, s));
  CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
  if (c->mixed) {
    launches += p_given ? mixed_prepare_P(c->mixed, a.P, a.ldc, s) : mixed_prepare(c->mixed, a, nocc, s);
  } else if (!p_given) {
    launch_pmat_f64(a, kpad, s);
    launches += 2;
  }
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaEventRecord(c->ev[2], s));
  float ms;
  CUDA_TRY(c, cudaEventSynchronize(c->ev[2]));
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]));
  t_dens += ms;
  for (int64_t p0 = 0; p0 < c->npts; p0 += c->chunk) {
    const int64_t nv = std::min<int64_t>(c->chunk, c->npts - p0);
    CUDA_TRY(c, cudaEventRecord(c->ev[3], s));
    if (c->mixed) launches += mixed_basis(c->mixed, a, p0, nv, gga, s);
    else { launch_basis_f64(a, p0, nv, gga, s); launches += 4; }
    CUDA_TRY(c, cudaEventRecord(c->ev[4], s));
    CUDA_TRY(c, cudaEventRecord(c->kev[0], s));
    if (c->mixed) launches += mixed_density(c->mixed, a, gga, s);
    else { launch_density_f64(a, gga, s); launches += 1; }
    CUDA_TRY(c, cudaEventRecord(c->kev[1], s));
    CUDA_TRY(c, cudaEventRecord(c->ev[5], s));
    launch_functional_f64(a, p0, nv, gga, s);
    launches += 2;
    CUDA_TRY(c, cudaEventRecord(c->ev[6], s));
    if (c->mixed) {
      launches += mixed_potential(c->mixed, a, gga, s, c->kev[2], c->kev[3]);
    } else {
      launch_zbuild_f64(a, gga, s);
      CUDA_TRY(c, cudaEventRecord(c->kev[2], s));
      launch_vpot_f64(a, gga, s);
      CUDA_TRY(c, cudaEventRecord(c->kev[3], s));
      launches += 2;
    }
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaEventRecord(c->ev[7], s));
    CUDA_TRY(c, cudaEventSynchronize(c->ev[7]));
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[3], c->ev[4])); t_basis += ms;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[4], c->ev[5])); t_dens += ms;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[5], c->ev[6])); t_func += ms;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[6], c->ev[7])); t_pot += ms;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->kev[0], c->kev[1])); t_x += ms;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->kev[2], c->kev[3])); t_v += ms;
  }
  CUDA_TRY(c, cudaEventRecord(c->ev[3], s));
  if (c->mixed) launches += mixed_pack(c->mixed, a, c->nbas, c->opt.ispin, 0, c->d_ham, s);
  else { launch_pack(a, c->nbas, c->opt.ispin, 0, c->d_ham, s); launches += 1; }
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaEventRecord(c->ev[4], s));
  CUDA_TRY(c, cudaEventSynchronize(c->ev[4]));
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]));
  t_pot += ms;
  if (c->mixed) {
    int flag = 0;
    if (mixed_error_flag(c->mixed, s, &flag) != PGXC_OK) return set_err(c, PGXC_ECUDA, "error-flag read failed");
    if (flag) return set_err(c, PGXC_ETIMEOUT, "a bounded tensor-core pipeline wait ran out");
  }
  if (tm) {
    tm->basis_ms = t_basis;
    tm->density_ms = t_dens;
    tm->functional_ms = t_func;
    tm->potential_ms = t_pot;
    tm->xgemm_ms = t_x;
    tm->vgemm_ms = t_v;
    tm->kernel_launches = launches;
  }
  return PGXC_OK;
}

static int check_build_args(pgxc_ctx* c, int32_t nbas, int32_t nocc, int32_t ispin, int64_t xc_length) {
  if (nbas != c->nbas) return set_err(c, PGXC_EINVAL, "nbas does not match the context's basis");
  if (ispin != c->opt.ispin) return set_err(c, PGXC_EINVAL, "ispin does not match the context");
  if (nocc < 0) return set_err(c, PGXC_EINVAL, "nocc < 0");
  if (xc_length != (int64_t)ispin * nbas * (nbas + 1) / 2)
    return set_err(c, PGXC_EINVAL, "xc_length must be ispin*nbas*(nbas+1)/2");
  return PGXC_OK;
}

static int host_build_tail(pgxc_ctx* c, int nocc, bool p_given, double* ham, int64_t xc_length, double* exc,
                           double* nel, pgxc_timings* tm);

int pgxc_build(pgxc_ctx* c, const double* C, const double* occ, int32_t nbas, int32_t nocc, int32_t ispin,
               double* ham, int64_t xc_length, double* exc, double* nel, pgxc_timings* tm) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  int st = check_build_args(c, nbas, nocc, ispin, xc_length);
  if (st) return st;
  if (!ham || !exc || !nel || (nocc > 0 && (!C || !occ))) return set_err(c, PGXC_EINVAL, "NULL output/input");
  if (!all_finite(C, (int64_t)nbas * nocc * ispin) || !all_finite(occ, (int64_t)nocc * ispin))
    return set_err(c, PGXC_ENONFINITE, "non-finite C or occ");
  CUDA_TRY(c, cudaSetDevice(c->device));
  if ((st = ensure_occ(c, nocc))) return st;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  CUDA_TRY(c, cudaEventRecord(c->ev[0], c->stream));
  if ((st = upload_orbitals(c, C, occ, nbas, nocc, kpad, cudaMemcpyHostToDevice))) return st;
  return host_build_tail(c, nocc, false, ham, xc_length, exc, nel, tm);
}

// The rest of a host-buffer build whose inputs were enqueued after c->ev[0]:
// the device build, the D2H of the packed matrix and of the two sums, added
// into the caller's arrays.
static int host_build_tail(pgxc_ctx* c, int nocc, bool p_given, double* ham, int64_t xc_length, double* exc,
                           double* nel, pgxc_timings* tm) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  int st;
  CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
  CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
  float h2d = 0;
  CUDA_TRY(c, cudaEventElapsedTime(&h2d, c->ev[0], c->ev[1]));
  pgxc_timings local{};
  if ((st = run_build(c, nocc, &local, p_given))) return st;
  // D2H of the packed matrix and the two sums
  cudaEvent_t e0 = c->ev[5], e1 = c->ev[6];
  CUDA_TRY(c, cudaEventRecord(e0, s));
  CUDA_TRY(c, cudaMemcpyAsync(c->h_ham, c->d_ham, sizeof(double) * xc_length, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(c->h_acc, a.acc, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaEventRecord(e1, s));
  CUDA_TRY(c, cudaEventSynchronize(e1));
  float d2h = 0, tot = 0;
  CUDA_TRY(c, cudaEventElapsedTime(&d2h, e0, e1));
  CUDA_TRY(c, cudaEventElapsedTime(&tot, c->ev[0], e1));
  if (!std::isfinite(c->h_acc[0]) || !std::isfinite(c->h_acc[2]))
    return set_err(c, PGXC_ENONFINITE, "non-finite E_xc or N_el");
  for (int64_t i = 0; i < xc_length; ++i) ham[i] += c->h_ham[i];
  *exc += c->h_acc[0];
  *nel += c->h_acc[2];
  if (tm) {
    *tm = local;
    tm->h2d_ms = h2d;
    tm->d2h_ms = d2h;
    tm->total_ms = tot;
  }
  return PGXC_OK;
}

int pgxc_build_density(pgxc_ctx* c, const double* P, int32_t nbas, int32_t ispin, double* ham, int64_t xc_length,
                       double* exc, double* nel, pgxc_timings* tm) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  int st = check_build_args(c, nbas, 0, ispin, xc_length);
  if (st) return st;
  if (!P || !ham || !exc || !nel) return set_err(c, PGXC_EINVAL, "NULL output/input");
  if (!all_finite(P, (int64_t)ispin * nbas * nbas)) return set_err(c, PGXC_ENONFINITE, "non-finite P");
  CUDA_TRY(c, cudaSetDevice(c->device));
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
  for (int sp = 0; sp < ispin; ++sp) {
    double* dP = sp ? c->P2 : a.P;
    CUDA_TRY(c, cudaMemsetAsync(dP, 0, sizeof(double) * a.ldc * a.ldc, s));
    CUDA_TRY(c, cudaMemcpy2DAsync(dP, sizeof(double) * a.ldc, P + (size_t)sp * nbas * nbas, sizeof(double) * nbas,
                                  sizeof(double) * nbas, nbas, cudaMemcpyHostToDevice, s));
  }
  return host_build_tail(c, 0, true, ham, xc_length, exc, nel, tm);
}

int pgxc_build_device(pgxc_ctx* c, const double* d_C, const double* d_occ, int32_t nbas, int32_t nocc, int32_t ispin,
                      double* d_ham, int64_t xc_length, double* d_exc_nel, pgxc_timings* tm) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  int st = check_build_args(c, nbas, nocc, ispin, xc_length);
  if (st) return st;
  if (!d_ham || !d_exc_nel || (nocc > 0 && (!d_C || !d_occ))) return set_err(c, PGXC_EINVAL, "NULL pointer");
  CUDA_TRY(c, cudaSetDevice(c->device));
  if ((st = ensure_occ(c, nocc))) return st;
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
  if ((st = upload_orbitals(c, d_C, d_occ, nbas, nocc, kpad, cudaMemcpyDeviceToDevice))) return st;
  pgxc_timings local{};
  if ((st = run_build(c, nocc, &local))) return st;
  CUDA_TRY(c, cudaMemcpyAsync(d_ham, c->d_ham, sizeof(double) * xc_length, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(d_exc_nel, a.acc, sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(d_exc_nel + 1, a.acc + 2, sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
  CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
  float tot = 0;
  CUDA_TRY(c, cudaEventElapsedTime(&tot, c->ev[0], c->ev[1]));
  if (tm) {
    *tm = local;
    tm->total_ms = tot;
  }
  return PGXC_OK;
}

// ---------------------------------------------------------------------------
// Post-SCF XC nuclear gradient (gradient.h): per chunk of points the basis
// values with Hessians, X = Phi P and Y_j = d_j Phi P (DMMA), the
// functional's coefficients per point, the orbital terms and the Becke weight
// term.  FP64, every layout; needs the raw grid (weights_are_raw, point_atom).
// The orbitals (kpad padded columns) are in the context's C1 buffers.
// ---------------------------------------------------------------------------
static int gradient_core(pgxc_ctx* c, int32_t nbas, int32_t ispin, int64_t kpad, double* grad, double* exc) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  launch_pmat_f64(a, kpad, s);
  if (ispin == 2) {
    BuildArgs b = a;
    b.C = c->C2;
    b.occ = c->occ2;
    b.P = c->P2;
    launch_pmat_f64(b, kpad, s);
  }
  // function -> atom
  std::vector<int> fatom((size_t)nbas);
  for (const DevShell& S : c->shells)
    for (int f = 0; f < (2 * S.l + 1) * S.nrad; ++f) fatom[(size_t)S.f0 + f] = S.atom;
  // chunk of points: 10 basis planes + 4 ispin X/Y planes of nbas x ld, under ~4 GB
  int64_t ld = 65536;
  while (ld > 128 && (double)(10 + 4 * ispin) * nbas * ld * 8.0 > 4.0e9) ld /= 2;
  const int64_t plane = (int64_t)nbas * ld;
  // The weight term needs only each point's w_raw f (ef, kept for the whole
  // grid: whole chunks of ld, which k_grad_points fills to the end) and runs after the chunk loop in launches of ldw points, as many as
  // its per-(atom, point) scratch of 3.5 natm ldw doubles allows under ~2 GB:
  // far more blocks than one basis chunk would give (its per-point loops over
  // atom pairs are long, and a few blocks per SM leave it latency-bound).
  int64_t ldw = round_up(c->npts, 128);
  while (ldw > 128 && 28.0 * c->natm * ldw > 2.0e9) ldw = round_up(ldw / 2, 128);
  // one scratch buffer, carved in 256-byte aligned pieces and kept in the
  // context for the next call (allocation and release of several GB per call
  // would cost more than the gradient's kernels)
  const size_t sizes[8] = {sizeof(double) * 10 * plane,         sizeof(double) * 4 * ispin * plane,
                           sizeof(double) * 5 * ispin * ld,      sizeof(double) * (size_t)round_up(c->npts, ld),
                           sizeof(double) * 3 * c->natm,         sizeof(double),
                           sizeof(double) * ((size_t)7 * c->natm * ldw / 2 + 1), sizeof(int) * (size_t)nbas};
  size_t offs[8], total = 0;
  for (int i = 0; i < 8; ++i) {
    offs[i] = total;
    total += (sizes[i] + 255) / 256 * 256;
  }
  if (total > c->grad_scr_bytes) {
    if (c->grad_scr) cudaFree(c->grad_scr);
    c->grad_scr = nullptr;
    c->grad_scr_bytes = 0;
    cudaError_t e = cudaMalloc(&c->grad_scr, total);
    if (e != cudaSuccess) {
      c->grad_scr = nullptr;
      return set_err(c, PGXC_ENOMEM, std::string("gradient scratch: ") + cudaGetErrorString(e));
    }
    c->grad_scr_bytes = total;
  }
  char* base = (char*)c->grad_scr;
  double* basis = (double*)(base + offs[0]);
  double* XY = (double*)(base + offs[1]);
  double* coef = (double*)(base + offs[2]);
  double* ef = (double*)(base + offs[3]);
  double* dgrad = (double*)(base + offs[4]);
  double* de = (double*)(base + offs[5]);
  double* wscr = (double*)(base + offs[6]);
  int* dfatom = (int*)(base + offs[7]);
  const bool mgga = PGXC_XC_IS_MGGA(c->opt.functional);
  const bool gga = PGXC_XC_IS_GGA(c->opt.functional) || mgga;
  int rc = PGXC_OK;
  do {
    if (cudaMemcpyAsync(dfatom, fatom.data(), sizeof(int) * nbas, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(dgrad, 0, sizeof(double) * 3 * c->natm, s) != cudaSuccess ||
        cudaMemsetAsync(de, 0, sizeof(double), s) != cudaSuccess) {
      rc = set_err(c, PGXC_ECUDA, "gradient set-up copies failed");
      break;
    }
    for (int64_t p0 = 0; p0 < c->npts && rc == PGXC_OK; p0 += ld) {
      const int64_t nv = std::min<int64_t>(ld, c->npts - p0);
      launch_basis_hess(a, p0, nv, ld, plane, basis, s);
      for (int sp = 0; sp < ispin; ++sp) {
        const double* P = sp ? c->P2 : a.P;
        // X (j = 0) or Y_j = (d_j Phi) P: (ld x nbas) = (ld x nbas)(nbas x nbas), P symmetric; the
        // Y_j only for meta-GGAs (tau and its terms), GGAs take V = W P after the coefficients
        for (int j = 0; j < (mgga ? 4 : 1); ++j)
          launch_grad_xy(basis + j * plane, ld, P, a.ldc, nbas, XY + (4 * sp + j) * plane, s);
      }
      if (rc) break;
      launch_grad_points(a.xc, c->opt.functional, gga, ispin, nbas, ld, p0, nv, a.w, c->d_wraw, basis, plane, XY,
                         coef, ef + p0, de, s);
      if (gga && !mgga)
        for (int sp = 0; sp < ispin; ++sp) {
          double* W = XY + (4 * sp + 1) * plane;
          launch_grad_w(nbas, ld, basis, plane, coef + (5 * sp + 1) * ld, W, s);
          launch_grad_xy(W, ld, sp ? c->P2 : a.P, a.ldc, nbas, XY + (4 * sp + 2) * plane, s);
        }
      launch_grad_orbital(gga, mgga, ispin, nbas, ld, p0, nv, c->natm, dfatom, c->d_owner, basis, plane, XY, coef,
                          dgrad, s);
      if (cudaGetLastError() != cudaSuccess) rc = set_err(c, PGXC_ECUDA, "gradient kernel launch failed");
    }
    if (rc) break;
    for (int64_t p0 = 0; p0 < c->npts; p0 += ldw) {
      const int64_t nv = std::min<int64_t>(ldw, c->npts - p0);
      launch_grad_weights(a.atoms, c->d_dist, c->natm, a.px, a.py, a.pz, c->d_owner, p0, nv, ldw, ef + p0, wscr,
                          dgrad, s);
    }
    if (cudaGetLastError() != cudaSuccess) rc = set_err(c, PGXC_ECUDA, "gradient kernel launch failed");
    if (rc) break;
    std::vector<double> hg((size_t)3 * c->natm);
    double he = 0.0;
    if (cudaMemcpyAsync(hg.data(), dgrad, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&he, de, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = set_err(c, PGXC_ECUDA, "gradient read-back failed");
      break;
    }
    for (size_t i = 0; i < hg.size(); ++i) {
      if (!std::isfinite(hg[i])) {
        rc = set_err(c, PGXC_ENONFINITE, "non-finite gradient");
        break;
      }
      grad[i] += hg[i];
    }
    if (exc) *exc += he;
  } while (false);
  cudaStreamSynchronize(s);
  return rc;
}

static int gradient_checks(pgxc_ctx* c, double* grad) {
  if (!grad) return set_err(c, PGXC_EINVAL, "NULL output");
  if (!c->d_owner)
    return set_err(c, PGXC_ENOTSUP, "the XC gradient needs a grid created with raw weights and point_atom "
                                    "(the grid moves with its atoms)");
  return PGXC_OK;
}

int pgxc_xc_gradient(pgxc_ctx* c, const double* C, const double* occ, int32_t nbas, int32_t nocc, int32_t ispin,
                     double* grad, double* exc) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  int st = check_build_args(c, nbas, nocc, ispin, (int64_t)ispin * nbas * (nbas + 1) / 2);
  if (st) return st;
  if ((st = gradient_checks(c, grad))) return st;
  if (nocc > 0 && (!C || !occ)) return set_err(c, PGXC_EINVAL, "NULL input");
  if (c->sym)
    return set_err(c, PGXC_EINVAL, "a context with pgxc_set_symmetry applied takes the irreps' orbitals: "
                                   "pgxc_xc_gradient_sym");
  if (!all_finite(C, (int64_t)nbas * nocc * ispin) || !all_finite(occ, (int64_t)nocc * ispin))
    return set_err(c, PGXC_ENONFINITE, "non-finite C or occ");
  CUDA_TRY(c, cudaSetDevice(c->device));
  if ((st = ensure_occ(c, nocc))) return st;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  if ((st = upload_orbitals(c, C, occ, nbas, nocc, kpad, cudaMemcpyHostToDevice))) return st;
  return gradient_core(c, nbas, ispin, kpad, grad, exc);
}

// ---------------------------------------------------------------------------
// Energies of several functionals on one density (post_scf_calc_xc_energy,
// modules/post_scf_module.f90:2204-2564, with the energy table of
// xc_func_get_exc, modules/xc_func.f90:1011-1200): one basis and density
// pass, one functional pass per requested functional, no potential.
// ---------------------------------------------------------------------------
int pgxc_xc_energies(pgxc_ctx* c, const double* C, const double* occ, int32_t nbas, int32_t nocc, int32_t ispin,
                     int32_t n, const int32_t* functionals, double* exc, double* nel) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  int st = check_build_args(c, nbas, nocc, ispin, (int64_t)ispin * nbas * (nbas + 1) / 2);
  if (st) return st;
  if (!c->screen) return set_err(c, PGXC_ENOTSUP, "pgxc_xc_energies needs a screened context (screen_threshold >= 0)");
  if (n < 1 || !functionals || !exc || (nocc > 0 && (!C || !occ))) return set_err(c, PGXC_EINVAL, "NULL or empty input");
  // grad rho (and the gradient planes) exist in GGA and meta-GGA contexts
  const bool gga = PGXC_XC_IS_GGA(c->opt.functional) || PGXC_XC_IS_MGGA(c->opt.functional);
  std::vector<XcConst> xcs((size_t)n);
  std::vector<int> ggas((size_t)n);
  bool tau = false;
  for (int i = 0; i < n; ++i) {
    const int f = functionals[i];
    if (f < PGXC_XC_VWN || f > PGXC_XC_LAST) return set_err(c, PGXC_EINVAL, "functional id out of range");
    const bool fg = PGXC_XC_IS_GGA(f) || PGXC_XC_IS_MGGA(f);
    if (fg && !gga)
      return set_err(c, PGXC_EINVAL, "a GGA energy needs a context created with a GGA functional (no grad rho)");
    tau = tau || PGXC_XC_IS_MGGA(f);
    if (!PGXC_XC_IS_MGGA(f)) xcs[i] = make_xc_const(f);
    ggas[i] = PGXC_XC_IS_GGA(f) ? 1 : 0;
  }
  if (tau) {  // meta-GGAs: the kinetic-energy density of the same orbitals
    std::string e;
    if ((st = screen_enable_tau(c->screen, e))) return set_err(c, st, e);
  }
  if (!all_finite(C, (int64_t)nbas * nocc * ispin) || !all_finite(occ, (int64_t)nocc * ispin))
    return set_err(c, PGXC_ENONFINITE, "non-finite C or occ");
  CUDA_TRY(c, cudaSetDevice(c->device));
  if ((st = ensure_occ(c, nocc))) return st;
  if (n > c->eacc_cap) {
    if ((st = dalloc(c, &c->d_eacc, (size_t)4 * n))) return st;
    c->eacc_cap = n;
  }
  double* d_acc = c->d_eacc;
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  if ((st = upload_orbitals(c, C, occ, nbas, nocc, kpad, cudaMemcpyHostToDevice))) return st;
  CUDA_TRY(c, cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), s));
  CUDA_TRY(c, cudaMemsetAsync(d_acc, 0, 4 * sizeof(double) * n, s));
  launch_pmat_f64(a, kpad, s);
  if (ispin == 2) {
    BuildArgs b = a;
    b.C = c->C2;
    b.occ = c->occ2;
    b.P = c->P2;
    launch_pmat_f64(b, kpad, s);
  }
  ScreenExtra x;
  x.xc = xcs.data();
  x.gga = ggas.data();
  x.fid = functionals;
  x.n = n;
  x.acc = d_acc;
  x.potential = false;
  x.tau = tau;
  std::string e;
  if ((st = screen_run(c->screen, a, c->P2, s, c->d_ham, nullptr, e, &x))) return set_err(c, st, e);
  std::vector<double> h((size_t)4 * n);
  CUDA_TRY(c, cudaMemcpyAsync(h.data(), d_acc, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  int flag = 0;
  if (screen_error_flag(c->screen, s, &flag) != PGXC_OK) return set_err(c, PGXC_ECUDA, "error-flag read failed");
  if (flag) return set_err(c, PGXC_ETIMEOUT, "a bounded tensor-core pipeline wait ran out");
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(h[4 * i])) return set_err(c, PGXC_ENONFINITE, "non-finite E_xc");
    exc[i] = h[4 * i];
  }
  if (nel) *nel = h[2];
  return PGXC_OK;
}

// ---------------------------------------------------------------------------
// Symmetry-adapted builds (n_irrep >= 1, partners >= 1): the irreps' orbitals
// are expanded into the C1 basis on the device, the C1 build runs on them,
// and the C1 potential is projected onto each irrep (symmetry.h).
// ---------------------------------------------------------------------------

int pgxc_set_symmetry(pgxc_ctx* c, const pgxc_symmetry* y) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  if (!y || y->n_irrep < 1 || !y->dims || !y->partners || y->nnz < 0 ||
      (y->nnz > 0 && (!y->irrep || !y->partner || !y->fn || !y->ao || !y->coef)))
    return set_err(c, PGXC_EINVAL, "symmetry: n_irrep >= 1, dims, partners and the nnz entries are required");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const int n = y->n_irrep;
  SymPlan* P = new (std::nothrow) SymPlan;
  if (!P) return set_err(c, PGXC_ENOMEM, "host allocation failed");
  P->dims.assign(y->dims, y->dims + n);
  P->partners.assign(y->partners, y->partners + n);
  P->ipbase.resize(n);
  P->pkofs.resize(n);
  std::vector<int> ip_irrep;
  std::vector<int64_t> colbase;
  int64_t ncol = 0;
  for (int i = 0; i < n; ++i) {
    const int d = P->dims[i], np = P->partners[i];
    if (d < 0 || np < 1) {
      delete P;
      return set_err(c, PGXC_EINVAL, "symmetry: dims >= 0 and partners >= 1 required");
    }
    P->ipbase[i] = P->nip;
    P->pkofs[i] = P->len;
    P->len += (int64_t)d * (d + 1) / 2;
    P->max_dim = std::max(P->max_dim, d);
    for (int p = 0; p < np; ++p) {
      ip_irrep.push_back(i);
      colbase.push_back(ncol);
      ncol += d;
    }
    P->nip += np;
  }
  struct E { int ip, fn, ao; double coef; };
  std::vector<E> ent((size_t)y->nnz);
  for (int64_t e = 0; e < y->nnz; ++e) {
    const int i = y->irrep[e], p = y->partner[e], f = y->fn[e], a = y->ao[e];
    if (i < 0 || i >= n || p < 0 || p >= P->partners[i] || f < 0 || f >= P->dims[i] || a < 0 || a >= c->nbas ||
        !std::isfinite(y->coef[e])) {
      delete P;
      return set_err(c, y->coef && !std::isfinite(y->coef[e]) ? PGXC_ENONFINITE : PGXC_EINVAL,
                     "symmetry: entry " + std::to_string(e) + " out of range or non-finite");
    }
    ent[e] = E{P->ipbase[i] + p, f, a, y->coef[e]};
  }
  // rows of U by (ip, C1 function): the orbital gather
  std::vector<E> rows = ent;
  std::stable_sort(rows.begin(), rows.end(), [](const E& x, const E& z) { return x.ip != z.ip ? x.ip < z.ip : x.ao < z.ao; });
  std::vector<int> grp_ip, grp_ao, row_fn;
  std::vector<int64_t> grp_ptr;
  std::vector<double> row_coef;
  for (size_t e = 0; e < rows.size(); ++e) {
    if (e == 0 || rows[e].ip != rows[e - 1].ip || rows[e].ao != rows[e - 1].ao) {
      grp_ip.push_back(rows[e].ip);
      grp_ao.push_back(rows[e].ao);
      grp_ptr.push_back((int64_t)e);
    }
    row_fn.push_back(rows[e].fn);
    row_coef.push_back(rows[e].coef);
  }
  grp_ptr.push_back((int64_t)rows.size());
  // columns of U by (ip, symmetry-adapted function): the potential gather
  std::vector<int64_t> col_ptr((size_t)ncol + 1, 0);
  for (const E& x : ent) ++col_ptr[colbase[x.ip] + x.fn + 1];
  for (int64_t k = 0; k < ncol; ++k) col_ptr[k + 1] += col_ptr[k];
  std::vector<int> col_ao(ent.size());
  std::vector<double> col_coef(ent.size());
  {
    std::vector<int64_t> fill(col_ptr.begin(), col_ptr.end() - 1);
    for (const E& x : ent) {
      const int64_t k = fill[colbase[x.ip] + x.fn]++;
      col_ao[k] = x.ao;
      col_coef[k] = x.coef;
    }
  }
  SymDev& D = P->dev;
  int *d_dims, *d_partners, *d_ipbase, *d_ip_irrep, *d_grp_ip, *d_grp_ao, *d_row_fn, *d_col_ao;
  int64_t *d_pkofs, *d_grp_ptr, *d_colbase, *d_col_ptr;
  double *d_row_coef, *d_col_coef;
  int st;
  if ((st = upload_vec(c, P->dims, &d_dims)) || (st = upload_vec(c, P->partners, &d_partners)) ||
      (st = upload_vec(c, P->ipbase, &d_ipbase)) || (st = upload_vec(c, P->pkofs, &d_pkofs)) ||
      (st = upload_vec(c, ip_irrep, &d_ip_irrep)) || (st = upload_vec(c, grp_ip, &d_grp_ip)) ||
      (st = upload_vec(c, grp_ao, &d_grp_ao)) || (st = upload_vec(c, grp_ptr, &d_grp_ptr)) ||
      (st = upload_vec(c, row_fn, &d_row_fn)) || (st = upload_vec(c, row_coef, &d_row_coef)) ||
      (st = upload_vec(c, colbase, &d_colbase)) || (st = upload_vec(c, col_ptr, &d_col_ptr)) ||
      (st = upload_vec(c, col_ao, &d_col_ao)) || (st = upload_vec(c, col_coef, &d_col_coef)) ||
      (st = dalloc(c, &P->d_ham, (size_t)c->opt.ispin * P->len)) || (st = dalloc(c, &P->d_nocc, (size_t)n)) ||
      (st = dalloc(c, &P->d_cofs, (size_t)c->opt.ispin * n)) || (st = dalloc(c, &P->d_col0, (size_t)P->nip))) {
    delete P;
    return st;
  }
  D.n_irrep = n;
  D.dims = d_dims;
  D.partners = d_partners;
  D.ipbase = d_ipbase;
  D.pkofs = d_pkofs;
  D.ip_irrep = d_ip_irrep;
  D.ngroups = (int)grp_ip.size();
  D.grp_ip = d_grp_ip;
  D.grp_ao = d_grp_ao;
  D.grp_ptr = d_grp_ptr;
  D.row_fn = d_row_fn;
  D.row_coef = d_row_coef;
  D.colbase = d_colbase;
  D.col_ptr = d_col_ptr;
  D.col_ao = d_col_ao;
  D.col_coef = d_col_coef;
  delete c->sym;
  c->sym = P;
  return PGXC_OK;
}

int pgxc_sym_xc_length(const pgxc_ctx* c, int64_t* xc_length) {
  if (!c || !xc_length) return set_err(nullptr, PGXC_EINVAL, "NULL argument");
  if (!c->sym) return set_err(nullptr, PGXC_EINVAL, "no symmetry set on this context");
  *xc_length = (int64_t)c->opt.ispin * c->sym->len;
  return PGXC_OK;
}

int pgxc_set_pseudo2d(pgxc_ctx* c, const int32_t* nblocks, const int32_t* first, const int32_t* half) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  SymPlan* P = c->sym;
  if (!P) return set_err(c, PGXC_EINVAL, "pgxc_set_pseudo2d needs pgxc_set_symmetry first");
  P->p2_pairs = P->p2_quads = 0;
  if (!nblocks) return PGXC_OK;
  const int n = P->dev.n_irrep;
  std::vector<Pseudo2dPair> pairs;
  std::vector<int64_t> qfirst(1, 0);
  int64_t b0 = 0;
  for (int i = 0; i < n; ++i) {
    const int nb = nblocks[i];
    if (nb < 0) return set_err(c, PGXC_EINVAL, "pseudo2d: negative block count");
    if (nb > 0 && (!first || !half)) return set_err(c, PGXC_EINVAL, "pseudo2d: first and half are required");
    for (int b = 0; b < nb; ++b) {
      const int64_t f = first[b0 + b], h = half[b0 + b];
      const int64_t next = b + 1 < nb ? first[b0 + b + 1] : P->dims[(size_t)i];
      if (f < 0 || h < 0 || f + 2 * h > next || (b + 1 < nb && next < f))
        return set_err(c, PGXC_EINVAL, "pseudo2d: blocks must be ascending, disjoint and inside the irrep");
    }
    // block pairs X >= Y in block order (the reference's unique-atom / l loops)
    for (int bx = 0; bx < nb; ++bx)
      for (int by = 0; by <= bx; ++by) {
        Pseudo2dPair q;
        q.pk = P->pkofs[(size_t)i];
        q.px = first[b0 + bx];
        q.hx = half[b0 + bx];
        q.py = first[b0 + by];
        q.hy = half[b0 + by];
        q.same = bx == by;
        const int64_t nq = q.same ? q.hx * (q.hx + 1) / 2 : q.hx * q.hy;
        if (nq == 0) continue;
        pairs.push_back(q);
        qfirst.push_back(qfirst.back() + nq);
      }
    b0 += nb;
  }
  CUDA_TRY(c, cudaSetDevice(c->device));
  int st;
  if ((st = dalloc(c, &P->d_p2, std::max<size_t>(pairs.size(), 1))) ||
      (st = dalloc(c, &P->d_p2first, qfirst.size())))
    return st;
  if (!pairs.empty())
    CUDA_TRY(c, cudaMemcpy(P->d_p2, pairs.data(), sizeof(Pseudo2dPair) * pairs.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(P->d_p2first, qfirst.data(), sizeof(int64_t) * qfirst.size(), cudaMemcpyHostToDevice));
  P->p2_pairs = (int64_t)pairs.size();
  P->p2_quads = qfirst.back();
  return PGXC_OK;
}

// The irreps' orbitals expanded into the C1 orbital buffers of the context
// (k_sym_orbitals): columns U_ip C_i with occupations occ_i / partners_i per
// (irrep, partner), both spins; *ntot_out = the number of C1 orbitals.
static int sym_expand(pgxc_ctx* c, const double* const* C, const double* const* occ, const int32_t* nocc,
                      int32_t ispin, int64_t* ntot_out) {
  SymPlan* P = c->sym;
  const int n = P->dev.n_irrep;
  int64_t ntot = 0, csa = 0;
  int nocc_max = 0;
  for (int i = 0; i < n; ++i) {
    if (nocc[i] < 0) return set_err(c, PGXC_EINVAL, "nocc < 0");
    const int64_t m = (int64_t)P->dims[i] * nocc[i] * ispin;
    if (nocc[i] > 0 && (!occ[i] || (m > 0 && !C[i]))) return set_err(c, PGXC_EINVAL, "NULL C or occ of an irrep");
    if ((m > 0 && !all_finite(C[i], m)) || (nocc[i] > 0 && !all_finite(occ[i], (int64_t)nocc[i] * ispin)))
      return set_err(c, PGXC_ENONFINITE, "non-finite C or occ");
    ntot += (int64_t)P->partners[i] * nocc[i];
    csa += m;
    nocc_max = std::max(nocc_max, (int)nocc[i]);
  }
  if (ntot > (1 << 30)) return set_err(c, PGXC_EINVAL, "too many orbitals");
  CUDA_TRY(c, cudaSetDevice(c->device));
  int st;
  if ((st = ensure_occ(c, (int)ntot))) return st;
  if (csa > P->csa_cap) {
    if ((st = dalloc(c, &P->d_Csa, (size_t)csa))) return st;
    P->csa_cap = csa;
  }
  // host layouts: the irreps' orbitals per spin, their offsets, the C1 column
  // of each (irrep, partner) block and the C1 occupations occ / partners
  const int64_t kpad = round_up(std::max<int64_t>(ntot, 1), 16);
  std::vector<double> hC((size_t)csa), hocc((size_t)ispin * kpad, 0.0);
  std::vector<int64_t> cofs((size_t)ispin * n), col0((size_t)P->nip);
  std::vector<int> hnocc(nocc, nocc + n);
  int64_t o = 0;
  for (int s = 0; s < ispin; ++s)
    for (int i = 0; i < n; ++i) {
      const int64_t m = (int64_t)P->dims[i] * nocc[i];
      cofs[(size_t)s * n + i] = o;
      if (m > 0) std::memcpy(hC.data() + o, C[i] + (size_t)s * m, sizeof(double) * m);
      o += m;
    }
  int64_t col = 0;
  for (int i = 0; i < n; ++i)
    for (int p = 0; p < P->partners[i]; ++p) {
      col0[P->ipbase[i] + p] = col;
      for (int s = 0; s < ispin; ++s)
        for (int k = 0; k < nocc[i]; ++k)
          hocc[(size_t)s * kpad + col + k] = occ[i][k + (size_t)nocc[i] * s] / P->partners[i];
      col += nocc[i];
    }
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  if (csa > 0) CUDA_TRY(c, cudaMemcpyAsync(P->d_Csa, hC.data(), sizeof(double) * csa, cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(P->d_cofs, cofs.data(), sizeof(int64_t) * cofs.size(), cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(P->d_nocc, hnocc.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(P->d_col0, col0.data(), sizeof(int64_t) * col0.size(), cudaMemcpyHostToDevice, s));
  for (int sp = 0; sp < ispin; ++sp) {
    double* dC = sp ? c->C2 : a.C;
    double* docc = sp ? c->occ2 : (double*)a.occ;
    CUDA_TRY(c, cudaMemsetAsync(dC, 0, sizeof(double) * kpad * a.ldc, s));
    CUDA_TRY(c, cudaMemcpyAsync(docc, hocc.data() + (size_t)sp * kpad, sizeof(double) * kpad, cudaMemcpyHostToDevice, s));
    launch_sym_orbitals(P->dev, P->d_Csa, P->d_cofs + (size_t)sp * n, P->d_nocc, P->d_col0, nocc_max, dC, a.ldc, s);
  }
  CUDA_TRY(c, cudaGetLastError());
  // the host staging vectors must outlive the asynchronous copies
  CUDA_TRY(c, cudaStreamSynchronize(s));
  *ntot_out = ntot;
  return PGXC_OK;
}

// The XC gradient of a symmetry-adapted context: the irreps' orbitals are
// expanded into C1 orbitals (the density is then the C1 one) and the C1
// gradient runs on the context's grid.  On a symmetry-reduced grid (the
// unique atoms' points, weights times n_equal_atoms, point_atom the first
// equal atom) this is the reference's grad_xc before post_scf_average_gradient.
int pgxc_xc_gradient_sym(pgxc_ctx* c, const double* const* C, const double* const* occ, const int32_t* nocc,
                         int32_t ispin, double* grad, double* exc) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  if (!c->sym) return set_err(c, PGXC_EINVAL, "pgxc_xc_gradient_sym needs pgxc_set_symmetry first");
  if (ispin != c->opt.ispin) return set_err(c, PGXC_EINVAL, "ispin does not match the context");
  if (!nocc || !C || !occ) return set_err(c, PGXC_EINVAL, "NULL input");
  int st = gradient_checks(c, grad);
  if (st) return st;
  CUDA_TRY(c, cudaSetDevice(c->device));
  int64_t ntot = 0;
  if ((st = sym_expand(c, C, occ, nocc, ispin, &ntot))) return st;
  const int64_t kpad = round_up(std::max<int64_t>(ntot, 1), 16);
  return gradient_core(c, (int32_t)c->nbas, ispin, kpad, grad, exc);
}

int pgxc_build_sym(pgxc_ctx* c, const double* const* C, const double* const* occ, const int32_t* nocc, int32_t ispin,
                   double* ham, int64_t xc_length, double* exc, double* nel, pgxc_timings* tm) {
  if (!c) return set_err(nullptr, PGXC_EINVAL, "ctx is NULL");
  SymPlan* P = c->sym;
  if (!P) return set_err(c, PGXC_EINVAL, "pgxc_build_sym needs pgxc_set_symmetry first");
  if (ispin != c->opt.ispin) return set_err(c, PGXC_EINVAL, "ispin does not match the context");
  if (xc_length != (int64_t)ispin * P->len)
    return set_err(c, PGXC_EINVAL, "xc_length must be ispin * sum_i dims_i (dims_i + 1) / 2");
  if (!ham || !exc || !nel || !nocc || !C || !occ) return set_err(c, PGXC_EINVAL, "NULL output/input");
  CUDA_TRY(c, cudaSetDevice(c->device));
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
  int64_t ntot = 0;
  int st;
  if ((st = sym_expand(c, C, occ, nocc, ispin, &ntot))) return st;
  CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
  CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
  float h2d = 0;
  CUDA_TRY(c, cudaEventElapsedTime(&h2d, c->ev[0], c->ev[1]));
  pgxc_timings local{};
  if ((st = run_build(c, (int)ntot, &local))) return st;
  cudaEvent_t e0 = c->ev[5], e1 = c->ev[6];
  CUDA_TRY(c, cudaEventRecord(e0, s));
  launch_sym_potential(P->dev, P->max_dim, ispin, c->d_ham, P->d_ham, s);
  launch_pseudo2d(P->d_p2, P->d_p2first, P->p2_pairs, P->p2_quads, ispin, P->d_ham, s);
  CUDA_TRY(c, cudaGetLastError());
  std::vector<double> hH((size_t)xc_length);
  if (xc_length > 0)
    CUDA_TRY(c, cudaMemcpyAsync(hH.data(), P->d_ham, sizeof(double) * xc_length, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(c->h_acc, a.acc, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaEventRecord(e1, s));
  CUDA_TRY(c, cudaEventSynchronize(e1));
  float d2h = 0, tot = 0;
  CUDA_TRY(c, cudaEventElapsedTime(&d2h, e0, e1));
  CUDA_TRY(c, cudaEventElapsedTime(&tot, c->ev[0], e1));
  if (!std::isfinite(c->h_acc[0]) || !std::isfinite(c->h_acc[2]))
    return set_err(c, PGXC_ENONFINITE, "non-finite E_xc or N_el");
  for (int64_t i = 0; i < xc_length; ++i) ham[i] += hH[i];
  *exc += c->h_acc[0];
  *nel += c->h_acc[2];
  if (tm) {
    *tm = local;
    tm->h2d_ms = h2d;
    tm->d2h_ms = d2h;
    tm->total_ms = tot;
    tm->kernel_launches += ispin + 1;
  }
  return PGXC_OK;
}

// ---------------------------------------------------------------------------
// Batched builds: the device builds of many screened contexts captured as the
// parallel branches of one CUDA graph.
// ---------------------------------------------------------------------------

// Enqueue the device build of a screened context on its stream without any
// synchronisation, event timing or host read (capturable): operands from
// device memory, the packed matrix and {E_xc, N_el} overwritten into d_ham,
// d_exc_nel.
static int enqueue_screened_build(pgxc_ctx* c, const double* d_C, const double* d_occ, int32_t nocc, double* d_ham,
                                  double* d_exc_nel) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  int st = upload_orbitals(c, d_C, d_occ, (int32_t)c->nbas, nocc, kpad, cudaMemcpyDeviceToDevice);
  if (st) return st;
  CUDA_TRY(c, cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), s));
  launch_pmat_f64(a, kpad, s);
  if (c->opt.ispin == 2) {
    BuildArgs b = a;
    b.C = c->C2;
    b.occ = c->occ2;
    b.P = c->P2;
    launch_pmat_f64(b, kpad, s);
  }
  CUDA_TRY(c, cudaGetLastError());
  std::string e;
  if ((st = screen_run(c->screen, a, c->P2, s, c->d_ham, nullptr, e))) return set_err(c, st, e);
  const int64_t len = (int64_t)c->opt.ispin * c->nbas * (c->nbas + 1) / 2;
  CUDA_TRY(c, cudaMemcpyAsync(d_ham, c->d_ham, sizeof(double) * len, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(d_exc_nel, a.acc, sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(d_exc_nel + 1, a.acc + 2, sizeof(double), cudaMemcpyDeviceToDevice, s));
  return PGXC_OK;
}

// A set member's share of a batch step (capturable): its orbitals uploaded,
// P formed and turned into digits, its accumulators zeroed.  The set's
// launches then build every member at once.
static int enqueue_set_member(pgxc_ctx* c, const double* d_C, const double* d_occ, int32_t nocc) {
  BuildArgs& a = c->a;
  cudaStream_t s = c->stream;
  const int64_t kpad = round_up(std::max(nocc, 1), 16);
  int st = upload_orbitals(c, d_C, d_occ, (int32_t)c->nbas, nocc, kpad, cudaMemcpyDeviceToDevice);
  if (st) return st;
  CUDA_TRY(c, cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), s));
  launch_pmat_f64(a, kpad, s);
  CUDA_TRY(c, cudaGetLastError());
  if (screen_set_prepare_member(c->screen, a.P, a.ldc, s)) return set_err(c, PGXC_ECUDA, "set member preparation");
  return PGXC_OK;
}

struct pgxc_batch {
  std::vector<pgxc_ctx*> ctx;
  ScreenSet* set = nullptr;  // the contexts' builds as one sequence of launches over all their tiles
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

void pgxc_batch_destroy(pgxc_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->set) screen_set_destroy(b->set);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {b->fork, b->t0, b->t1})
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int pgxc_batch_create(pgxc_ctx* const* ctx, int32_t n, const double* const* d_C, const double* const* d_occ,
                      const int32_t* nocc, double* const* d_ham, double* const* d_exc_nel, pgxc_batch** out) {
  return pgxc_batch_create_chunked(ctx, n, d_C, d_occ, nocc, d_ham, d_exc_nel, 0, out);
}

int pgxc_batch_is_set(const pgxc_batch* b, int32_t* is_set) {
  if (!b || !is_set) return set_err(nullptr, PGXC_EINVAL, "NULL argument");
  *is_set = b->set != nullptr;
  return PGXC_OK;
}

int pgxc_batch_create_chunked(pgxc_ctx* const* ctx, int32_t n, const double* const* d_C,
                              const double* const* d_occ, const int32_t* nocc, double* const* d_ham,
                              double* const* d_exc_nel, int64_t max_chunk_points, pgxc_batch** out) {
  if (!out) return set_err(nullptr, PGXC_EINVAL, "out is NULL");
  *out = nullptr;
  if (!ctx || n <= 0 || !d_C || !d_occ || !nocc || !d_ham || !d_exc_nel)
    return set_err(nullptr, PGXC_EINVAL, "batch: NULL array or n <= 0");
  std::vector<pgxc_ctx*> seen;
  for (int32_t i = 0; i < n; ++i) {
    pgxc_ctx* c = ctx[i];
    if (!c) return set_err(nullptr, PGXC_EINVAL, "batch: NULL context");
    if (!c->screen) return set_err(nullptr, PGXC_ENOTSUP, "batch: every context must use the screened layout");
    if (c->device != ctx[0]->device) return set_err(nullptr, PGXC_EINVAL, "batch: contexts on different devices");
    if (nocc[i] < 0 || (nocc[i] > 0 && (!d_C[i] || !d_occ[i])) || !d_ham[i] || !d_exc_nel[i])
      return set_err(nullptr, PGXC_EINVAL, "batch: bad operand of context " + std::to_string(i));
    if (std::find(seen.begin(), seen.end(), c) != seen.end())
      return set_err(nullptr, PGXC_EINVAL, "batch: a context appears twice");
    seen.push_back(c);
  }
  pgxc_batch* b = new pgxc_batch();
  b->ctx.assign(ctx, ctx + n);
  b->device = ctx[0]->device;
  b->join.assign((size_t)n, nullptr);
  auto fail = [&](int st, const std::string& msg) {
    pgxc_batch_destroy(b);
    return set_err(nullptr, st, msg);
  };
  cudaError_t ce = cudaSetDevice(b->device);
  for (int32_t i = 0; i < n && ce == cudaSuccess; ++i) {
    if (int st = ensure_occ(ctx[i], nocc[i])) return fail(st, "batch: context " + std::to_string(i) + ": " + ctx[i]->err);
    ce = cudaStreamSynchronize(ctx[i]->stream);  // nothing of the context is pending when the capture starts
  }
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreate(&b->t0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&b->t1);
  for (int32_t i = 0; i < n && ce == cudaSuccess; ++i) ce = cudaEventCreateWithFlags(&b->join[(size_t)i], cudaEventDisableTiming);
  if (ce != cudaSuccess) return fail(PGXC_ECUDA, std::string("batch: ") + cudaGetErrorString(ce));
  // Contexts that all use the screened INT8 closed-shell layout run as one
  // set: per chunk of their concatenated tiles one launch per kernel.
  bool as_set = true;
  for (int32_t i = 0; i < n && as_set; ++i)
    as_set = ctx[i]->opt.precision == PGXC_PREC_MIXED_INT8 && !ctx[i]->sym && ctx[i]->a.sa.identity &&
             screen_set_eligible(ctx[i]->screen);
  if (as_set) {
    std::vector<SetMember> mem;
    for (int32_t i = 0; i < n; ++i)
      mem.push_back({ctx[i]->screen, &ctx[i]->a, ctx[i]->opt.functional, d_ham[i], d_exc_nel[i]});
    std::string e;
    if (int st = screen_set_create(&b->set, mem, std::max<int64_t>(max_chunk_points, 0), b->stream, e))
      return fail(st, "batch: " + e);
  }
  // fork from the batch stream into every context's stream, join back
  ce = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
  if (ce != cudaSuccess) return fail(PGXC_ECUDA, std::string("batch: begin capture: ") + cudaGetErrorString(ce));
  int st = PGXC_OK;
  std::string msg;
  ce = cudaEventRecord(b->fork, b->stream);
  for (int32_t i = 0; i < n && ce == cudaSuccess && st == PGXC_OK; ++i) {
    pgxc_ctx* c = ctx[i];
    ce = cudaStreamWaitEvent(c->stream, b->fork, 0);
    if (ce != cudaSuccess) break;
    if ((st = b->set ? enqueue_set_member(c, d_C[i], d_occ[i], nocc[i])
                     : enqueue_screened_build(c, d_C[i], d_occ[i], nocc[i], d_ham[i], d_exc_nel[i]))) {
      msg = "batch: context " + std::to_string(i) + ": " + c->err;
      break;
    }
    ce = cudaEventRecord(b->join[(size_t)i], c->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->join[(size_t)i], 0);
  }
  if (b->set && st == PGXC_OK && ce == cudaSuccess) {
    std::string e;
    if ((st = screen_set_run(b->set, b->stream, e))) msg = "batch: " + e;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce_end = cudaStreamEndCapture(b->stream, &g);  // always ends the capture
  if (st == PGXC_OK && ce == cudaSuccess) ce = ce_end;
  if (st != PGXC_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return fail(st != PGXC_OK ? st : PGXC_ECUDA, st != PGXC_OK ? msg : std::string("batch: capture: ") + cudaGetErrorString(ce));
  }
  b->graph = g;
  ce = cudaGraphInstantiate(&b->exec, g, 0);
  if (ce != cudaSuccess) return fail(PGXC_ECUDA, std::string("batch: instantiate: ") + cudaGetErrorString(ce));
  *out = b;
  return PGXC_OK;
}

int pgxc_batch_run(pgxc_batch* b, double* ms) {
  if (!b) return set_err(nullptr, PGXC_EINVAL, "batch is NULL");
  CUDA_TRY(nullptr, cudaSetDevice(b->device));
  CUDA_TRY(nullptr, cudaEventRecord(b->t0, b->stream));
  CUDA_TRY(nullptr, cudaGraphLaunch(b->exec, b->stream));
  CUDA_TRY(nullptr, cudaEventRecord(b->t1, b->stream));
  CUDA_TRY(nullptr, cudaEventSynchronize(b->t1));
  if (ms) {
    float f = 0;
    CUDA_TRY(nullptr, cudaEventElapsedTime(&f, b->t0, b->t1));
    *ms = f;
  }
  if (b->set) {
    int flag = 0;
    if (screen_set_error_flag(b->set, b->stream, &flag) != PGXC_OK)
      return set_err(nullptr, PGXC_ECUDA, "batch: error-flag read failed");
    if (flag) return set_err(nullptr, PGXC_ETIMEOUT, "batch: a bounded tensor-core pipeline wait ran out");
  }
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    int flag = 0;
    if (screen_error_flag(b->ctx[i]->screen, b->ctx[i]->stream, &flag) != PGXC_OK)
      return set_err(nullptr, PGXC_ECUDA, "batch: error-flag read failed");
    if (flag)
      return set_err(nullptr, PGXC_ETIMEOUT,
                     "batch: context " + std::to_string(i) + ": a bounded tensor-core pipeline wait ran out");
  }
  return PGXC_OK;
}

int pgxc_batch_stats(const pgxc_batch* b, int64_t* kernel_nodes, int64_t* nodes) {
  if (!b || !kernel_nodes || !nodes) return set_err(nullptr, PGXC_EINVAL, "NULL argument");
  size_t n = 0;
  CUDA_TRY(nullptr, cudaGraphGetNodes(b->graph, nullptr, &n));
  std::vector<cudaGraphNode_t> v(n);
  if (n) CUDA_TRY(nullptr, cudaGraphGetNodes(b->graph, v.data(), &n));
  int64_t k = 0;
  for (cudaGraphNode_t node : v) {
    cudaGraphNodeType t;
    CUDA_TRY(nullptr, cudaGraphNodeGetType(node, &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  *kernel_nodes = k;
  *nodes = (int64_t)n;
  return PGXC_OK;
}

int pgxc_grid_weights(const pgxc_ctx* cc, double* w_out, int64_t npts) {
  pgxc_ctx* c = const_cast<pgxc_ctx*>(cc);
  if (!c || !w_out) return set_err(c, PGXC_EINVAL, "NULL argument");
  if (npts != c->npts) return set_err(c, PGXC_EINVAL, "npts mismatch");
  CUDA_TRY(c, cudaSetDevice(c->device));
  CUDA_TRY(c, cudaMemcpy(w_out, c->a.w, sizeof(double) * npts, cudaMemcpyDeviceToHost));
  return PGXC_OK;
}

int pgxc_orbital_calculate(pgxc_ctx* c, int64_t npts, const double* pts, double* phi, double* grads) {
  if (!c || !pts || !phi || npts < 0) return set_err(c, PGXC_EINVAL, "bad arguments");
  if (npts == 0) return PGXC_OK;
  CUDA_TRY(c, cudaSetDevice(c->device));
  const int64_t nb = c->nbas;
  double *dp, *dphi, *dg = nullptr;
  // temporary buffers: owned by this call
  CUDA_TRY(c, cudaMalloc(&dp, sizeof(double) * 3 * npts));
  cudaError_t e = cudaMalloc(&dphi, sizeof(double) * nb * npts);
  if (e == cudaSuccess && grads) e = cudaMalloc(&dg, sizeof(double) * 3 * nb * npts);
  int st = PGXC_OK;
  if (e != cudaSuccess) st = set_err(c, PGXC_ENOMEM, "cudaMalloc failed in pgxc_orbital_calculate");
  if (!st) {
    cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * npts, cudaMemcpyHostToDevice, c->stream);
    launch_basis_points_f64(c->a, dp, dp + npts, dp + 2 * npts, npts, npts, dphi, grads ? dg : nullptr,
                            grads ? dg + nb * npts : nullptr, grads ? dg + 2 * nb * npts : nullptr, c->stream);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) st = set_err(c, PGXC_ECUDA, std::string("basis kernel: ") + cudaGetErrorString(e));
  }
  if (!st) {
    // device layout [f][p] is already phi(npts, nbas) column-major
    cudaMemcpy(phi, dphi, sizeof(double) * nb * npts, cudaMemcpyDeviceToHost);
    if (grads) {
      // device [c][f][p] -> Fortran (npts, 3, nbas): element (p, c, f) at p + npts*(c + 3 f)
      std::vector<double> tmp((size_t)3 * nb * npts);
      cudaMemcpy(tmp.data(), dg, sizeof(double) * 3 * nb * npts, cudaMemcpyDeviceToHost);
      for (int cc2 = 0; cc2 < 3; ++cc2)
        for (int64_t f = 0; f < nb; ++f)
          std::memcpy(grads + npts * (cc2 + 3 * f), tmp.data() + (cc2 * nb + f) * npts, sizeof(double) * npts);
    }
  }
  cudaFree(dp);
  cudaFree(dphi);
  if (dg) cudaFree(dg);
  return st;
}

int pgxc_xc_functionals_mgga(int32_t functional, int32_t ispin, int64_t n, const double* rho, const double* gam,
                             const double* tau, double* f, double* fr, double* fg, double* ft) {
  if (!PGXC_XC_IS_MGGA(functional)) return set_err(nullptr, PGXC_EINVAL, "not a meta-GGA functional id");
  if (ispin != 1 && ispin != 2) return set_err(nullptr, PGXC_EINVAL, "ispin must be 1 or 2");
  if (n < 0 || !rho || !gam || !tau || !f || !fr || !fg || !ft) return set_err(nullptr, PGXC_EINVAL, "bad arguments");
  if (n == 0) return PGXC_OK;
  int st = check_device(nullptr, -1);
  if (st) return st;
  const int64_t ng = 2 * ispin - 1;
  const int64_t cols = 2 * (2 * ispin + ng) + 1;  // in: rho, gam, tau; out: f, fr, fg, ft
  double* d;
  if (cudaMalloc(&d, sizeof(double) * cols * n) != cudaSuccess) return set_err(nullptr, PGXC_ENOMEM, "cudaMalloc");
  double *drho = d, *dgam = drho + ispin * n, *dtau = dgam + ng * n, *df = dtau + ispin * n, *dfr = df + n,
         *dfg = dfr + ispin * n, *dft = dfg + ng * n;
  cudaError_t e = cudaMemcpy(drho, rho, sizeof(double) * ispin * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dgam, gam, sizeof(double) * ng * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dtau, tau, sizeof(double) * ispin * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    launch_xc_points_mgga(functional, ispin, n, drho, dgam, dtau, df, dfr, dfg, dft, 0);
    e = cudaDeviceSynchronize();
  }
  if (e == cudaSuccess) e = cudaMemcpy(f, df, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(fr, dfr, sizeof(double) * ispin * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(fg, dfg, sizeof(double) * ng * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(ft, dft, sizeof(double) * ispin * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_err(nullptr, PGXC_ECUDA, cudaGetErrorString(e));
  return PGXC_OK;
}

int pgxc_xc_functionals(int32_t functional, int32_t ispin, int64_t n, const double* rho, const double* gam, double* f,
                        double* fr, double* fg) {
  if (functional < PGXC_XC_VWN || functional > PGXC_XC_LAST) return set_err(nullptr, PGXC_EINVAL, "functional");
  if (PGXC_XC_IS_MGGA(functional)) return set_err(nullptr, PGXC_EINVAL, "a meta-GGA needs tau: pgxc_xc_functionals_mgga");
  if (ispin != 1 && ispin != 2) return set_err(nullptr, PGXC_EINVAL, "ispin must be 1 or 2");
  if (n < 0 || !rho || !f || !fr) return set_err(nullptr, PGXC_EINVAL, "bad arguments");
  const bool gga = PGXC_XC_IS_GGA(functional);
  if (gga && (!gam || !fg)) return set_err(nullptr, PGXC_EINVAL, "PBE needs gam and fg");
  if (n == 0) return PGXC_OK;
  int st = check_device(nullptr, -1);
  if (st) return st;
  const int64_t ng = 2 * ispin - 1;  // columns of gam and fg
  // device layout: rho (ispin), gam (ng), f (1), fr (ispin), fg (ng) columns of n
  const int64_t cols = 2 * ispin + 2 * ng + 1;
  double* d;
  if (cudaMalloc(&d, sizeof(double) * cols * n) != cudaSuccess) return set_err(nullptr, PGXC_ENOMEM, "cudaMalloc");
  double *drho = d, *dgam = d + ispin * n, *df = dgam + ng * n, *dfr = df + n, *dfg = dfr + ispin * n;
  cudaMemcpy(drho, rho, sizeof(double) * ispin * n, cudaMemcpyHostToDevice);
  if (gga) cudaMemcpy(dgam, gam, sizeof(double) * ng * n, cudaMemcpyHostToDevice);
  launch_xc_points(functional, ispin, n, drho, dgam, df, dfr, dfg, 0);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    cudaMemcpy(f, df, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(fr, dfr, sizeof(double) * ispin * n, cudaMemcpyDeviceToHost);
    if (gga) cudaMemcpy(fg, dfg, sizeof(double) * ng * n, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (e != cudaSuccess) return set_err(nullptr, PGXC_ECUDA, cudaGetErrorString(e));
  return PGXC_OK;
}

int pgxc_becke_weights(const pgxc_geometry* geo, int64_t npts, const double* pts, const int32_t* point_atom,
                       double* w_out) {
  if (!geo || geo->natoms <= 0 || !geo->coords || npts < 0 || !pts || !point_atom || !w_out)
    return set_err(nullptr, PGXC_EINVAL, "bad arguments");
  for (int64_t i = 0; i < npts; ++i)
    if (point_atom[i] < 0 || point_atom[i] >= geo->natoms) return set_err(nullptr, PGXC_EINVAL, "point_atom range");
  if (npts == 0) return PGXC_OK;
  int st = check_device(nullptr, -1);
  if (st) return st;
  const int natm = geo->natoms;
  double *d = nullptr, *datoms = nullptr, *ddist = nullptr;
  int* downer = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(double) * 4 * npts);
  if (e == cudaSuccess) e = cudaMalloc(&datoms, sizeof(double) * 3 * natm);
  if (e == cudaSuccess) e = cudaMalloc(&ddist, 2 * sizeof(double) * natm * natm);
  if (e == cudaSuccess) e = cudaMalloc(&downer, sizeof(int) * npts);
  const bool oom = e == cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaMemcpy(d, pts, sizeof(double) * 3 * npts, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(datoms, geo->coords, sizeof(double) * 3 * natm, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(downer, point_atom, sizeof(int) * npts, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_becke(datoms, ddist, natm, d, d + npts, d + 2 * npts, downer, npts, d + 3 * npts, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(w_out, d + 3 * npts, sizeof(double) * npts, cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(datoms);
  cudaFree(ddist);
  cudaFree(downer);
  if (e != cudaSuccess)
    return set_err(nullptr, oom ? PGXC_ENOMEM : PGXC_ECUDA, std::string("Becke weights: ") + cudaGetErrorString(e));
  return PGXC_OK;
}

}  // extern "C"
