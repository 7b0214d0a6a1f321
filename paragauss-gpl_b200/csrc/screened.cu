// screened.cu -- planning and FP64 kernels of the screened (tile-sparse) XC build.
//
// Per geometry (screen_create):
//   Morton order of the grid, tiles of 128 points (padded with weight-0 copies);
//   k_tile_atom_d2    smallest squared distance of each tile to each atom;
//   host plan         per tile the listed functions (slots, padded to 32), the
//                     basis work items (tile, shell, radial mask) and chunks.
// Per build (screen_run), per chunk of tiles:
//   k_basis_items     phi, grad phi of listed functions only     [K1]
//   k_pad_zero        zero the padding slots at the end of each tile's list
//   k_sdensity        X = phi_t P[S_t, S_t] on DMMA, P gathered by cp.async,
//                     fused rho, grad rho                          [K3]
//   k_functional      (kernels_fp64.cu)                            [K2]
//   k_szbuild         Z = A phi (+ B . grad phi)
//   k_svpot           H[S_t, S_t] += Z_t^T phi_t on DMMA, scatter-added into
//                     the full matrix with FP64 atomics            [K4]
// then k_spack packs V (LDA: H; GGA: H + H^T, the symmetrisation of
// modules/xc_hamiltonian.f90:1559-1566) into the tristore order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "basis.cuh"
#include "dgemm.cuh"
#include "grid.h"
#include "kernels.h"
#include "screened.h"
#include "screened_mixed.h"
#include "screened_plan.h"

namespace pgxc {

namespace {

template <typename T>
cudaError_t sp_alloc(ScreenPlan* sp, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) {
    sp->allocs.push_back(q);
    *p = (T*)q;
  }
  return e;
}

// ---------------------------------------------------------------------------
// planning kernels
// ---------------------------------------------------------------------------
__global__ void k_gather_points(const int64_t* __restrict__ perm, int64_t nq, const double* __restrict__ px,
                                const double* __restrict__ py, const double* __restrict__ pz,
                                const double* __restrict__ w, double* __restrict__ qx, double* __restrict__ qy,
                                double* __restrict__ qz, double* __restrict__ qw) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  int64_t i = perm[q];
  double wt = 0.0;
  if (i >= 0) wt = w[i];
  else i = perm[q & ~(int64_t)127];  // padding: a weight-0 copy of the tile's first point
  qx[q] = px[i];
  qy[q] = py[i];
  qz[q] = pz[i];
  qw[q] = wt;
}

// d2[t][a] = min over the tile's points of |r - R_a|^2, rounded down to float
__global__ void __launch_bounds__(128) k_tile_atom_d2(const double* __restrict__ qx, const double* __restrict__ qy,
                                                      const double* __restrict__ qz, const double* __restrict__ atoms,
                                                      int natm, float* __restrict__ d2) {
  __shared__ float red[4];
  const int64_t t = blockIdx.x;
  const int64_t q = t * 128 + threadIdx.x;
  const double x = qx[q], y = qy[q], z = qz[q];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int a = 0; a < natm; ++a) {
    const double dx = x - atoms[3 * a], dy = y - atoms[3 * a + 1], dz = z - atoms[3 * a + 2];
    float f = __double2float_rd(dx * dx + dy * dy + dz * dz);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f = fminf(f, __shfl_xor_sync(0xffffffffu, f, o));
    if (lane == 0) red[warp] = f;
    __syncthreads();
    if (threadIdx.x == 0) d2[t * natm + a] = fminf(fminf(red[0], red[1]), fminf(red[2], red[3]));
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// FP64 kernels
// ---------------------------------------------------------------------------
// Zero the padding slots of each tile (the slots after its listed
// functions: tso[t] + listed[t] .. tso[t+1]).  grid = chunk tiles.
template <bool GGA, typename GT = double>
__global__ void __launch_bounds__(128) k_pad_zero(const int64_t* __restrict__ tso, const int* __restrict__ listed,
                                                  int64_t t0, int64_t s0, double* __restrict__ phi,
                                                  GT* __restrict__ gx, GT* __restrict__ gy,
                                                  GT* __restrict__ gz) {
  const int64_t t = t0 + blockIdx.x;
  const int64_t r0 = tso[t] - s0 + listed[t], r1 = tso[t + 1] - s0;
  for (int64_t e = r0 * 128 + threadIdx.x; e < r1 * 128; e += 128) {
    phi[e] = 0.0;
    if (GGA) {
      gx[e] = (GT)0;
      gy[e] = (GT)0;
      gz[e] = (GT)0;
    }
  }
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;  // 0: fill with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}

// B slab of the density GEMM: element (k, n) = P[fn(k0+k)][fn(n0+n)], zero
// where a slot is padding or n0+n >= n_valid.
__device__ __forceinline__ void load_gslab(double* s, const double* __restrict__ P, int64_t ldc,
                                           const int* __restrict__ sfn, int nvalid, int n0, int k0) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int c = t + i * kGemmThreads;
    const int k = c >> 6, nn = c & 63;
    const int fk = sfn[k0 + k];
    const int col = n0 + nn;
    const int fn = col < nvalid ? sfn[col] : -1;
    const bool ok = fk >= 0 && fn >= 0;
    cp_async8(s + OpTile<false, 64>::idx(nn, k), ok ? P + (int64_t)fk * ldc + fn : P, ok);
  }
}

// K3 (screened): CTA = (tile, half of its 128 points); loops over 64-wide
// blocks of the tile's slots.  The tile's slot -> function list is kept in
// shared memory after the GEMM stages.
template <bool GGA>
__global__ void __launch_bounds__(kGemmThreads) k_sdensity(const double* __restrict__ phi,
                                                          const double* __restrict__ gx,
                                                          const double* __restrict__ gy,
                                                          const double* __restrict__ gz,
                                                          const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
                                                          const int* __restrict__ slot_fn,
                                                          const double* __restrict__ P, int64_t ldc,
                                                          double* __restrict__ rho, double* __restrict__ grx,
                                                          double* __restrict__ gry, double* __restrict__ grz) {
  extern __shared__ double smem[];
  constexpr int EA = OpTile<false, 64>::kElems, EB = OpTile<false, 64>::kElems;
  double* sA = smem;
  double* sB = smem + kStages * EA;
  int* sfn = reinterpret_cast<int*>(smem + kStages * (EA + EB));
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int m0 = blockIdx.y * 64;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sfn[i] = slot_fn[tso[t] + i];
  __syncthreads();
  const double* A = phi + sb * 128;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
  const int fr = lane >> 2, fk = lane & 3;
  const int nslab = n / kBK;
  double rp[4][2] = {}, gp[3][4][2] = {};
  for (int n0 = 0; n0 < n; n0 += 64) {
    Acc acc;
    acc.zero();
#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
      if (s < nslab) {
        load_slab<false>(sA + s * EA, A, 128, m0, (int64_t)s * kBK);
        load_gslab(sB + s * EB, P, ldc, sfn, n, n0, s * kBK);
      }
      cp_async_commit();
    }
    for (int it = 0; it < nslab; ++it) {
      cp_async_wait<kStages - 2>();
      __syncthreads();
      {
        const int nx = it + kStages - 1;
        if (nx < nslab) {
          const int st = nx % kStages;
          load_slab<false>(sA + st * EA, A, 128, m0, (int64_t)nx * kBK);
          load_gslab(sB + st * EB, P, ldc, sfn, n, n0, nx * kBK);
        }
        cp_async_commit();
      }
      const double* a_s = sA + (it % kStages) * EA;
      const double* b_s = sB + (it % kStages) * EB;
#pragma unroll
      for (int kk = 0; kk < kBK; kk += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) af[i] = a_s[OpTile<false, 64>::idx(wm0 + i * 8 + fr, kk + fk)];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = b_s[OpTile<false, 64>::idx(wn0 + j * 8 + fr, kk + fk)];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc.v[i][j], af[i], bf[j]);
      }
    }
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = m0 + wm0 + i * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = n0 + wn0 + j * 8 + 2 * (lane & 3) + e;
          if (c < n) {
            const double x = acc.v[i][j][e];
            const int64_t o = (sb + c) * 128 + r;
            rp[i][e] += x * phi[o];
            if (GGA) {
              gp[0][i][e] += x * gx[o];
              gp[1][i][e] += x * gy[o];
              gp[2][i][e] += x * gz[o];
            }
          }
        }
    }
  }
  // reduce the 4 lanes of a row, then the two column-warps through smem
  double* red = smem;  // [2 warps-n][4 quantities][64 rows]
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double v[4];
    v[0] = rp[i][0] + rp[i][1];
    if (GGA) {
      v[1] = gp[0][i][0] + gp[0][i][1];
      v[2] = gp[1][i][0] + gp[1][i][1];
      v[3] = gp[2][i][0] + gp[2][i][1];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q > 0 && !GGA) break;
      v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
      v[q] += __shfl_xor_sync(0xffffffffu, v[q], 2);
      if ((lane & 3) == 0) red[((warp & 1) * 4 + q) * 64 + wm0 + i * 8 + (lane >> 2)] = v[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    const int r = threadIdx.x;
    const int64_t o = (int64_t)blockIdx.x * 128 + m0 + r;
    rho[o] = red[0 * 64 + r] + red[4 * 64 + r];
    if (GGA) {
      grx[o] = 2.0 * (red[1 * 64 + r] + red[5 * 64 + r]);
      gry[o] = 2.0 * (red[2 * 64 + r] + red[6 * 64 + r]);
      grz[o] = 2.0 * (red[3 * 64 + r] + red[7 * 64 + r]);
    }
  }
}

// Z[s][p] = A[p] phi[s][p] (+ B[p] . grad phi[s][p]) over the chunk's slots
template <bool GGA>
__global__ void k_szbuild(int64_t nslots, const int* __restrict__ slot_tile, int64_t t0,
                          const double* __restrict__ phi, const double* __restrict__ gx,
                          const double* __restrict__ gy, const double* __restrict__ gz,
                          const double* __restrict__ A, const double* __restrict__ Bx,
                          const double* __restrict__ By, const double* __restrict__ Bz, double* __restrict__ Z) {
  const int64_t total = nslots * 128;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = ((int64_t)slot_tile[e >> 7] - t0) * 128 + (e & 127);
    double z = A[p] * phi[e];
    if (GGA) z += Bx[p] * gx[e] + By[p] * gy[e] + Bz[p] * gz[e];
    Z[e] = z;
  }
}

// (I, J) of pair q of the tile's nb 64-slot blocks: all nb^2 (GGA) or I <= J (LDA)
__device__ __forceinline__ void pair_of(int q, int nb, bool all, int& I, int& J) {
  if (all) {
    I = q / nb;
    J = q % nb;
    return;
  }
  I = 0;
  while (q >= nb - I) {
    q -= nb - I;
    ++I;
  }
  J = I + q;
}

// K4 (screened): H[fn_i][fn_j] += sum_p Z[i][p] phi[j][p] for the slots i, j
// of one tile; LDA keeps fn_i <= fn_j only (H is symmetric), GGA the whole
// square (V = H + H^T in k_spack).
template <bool GGA>
__global__ void __launch_bounds__(kGemmThreads) k_svpot(const double* __restrict__ phi, const double* __restrict__ Z,
                                                       const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
                                                       const int* __restrict__ slot_fn, double* __restrict__ V,
                                                       int64_t ldv) {
  extern __shared__ double smem[];
  constexpr int kGemmDoubles = kStages * (OpTile<true, 64>::kElems + OpTile<true, 64>::kElems);
  int* sfn = reinterpret_cast<int*>(smem + kGemmDoubles);
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  for (int i = threadIdx.x; i < n; i += blockDim.x) sfn[i] = slot_fn[tso[t] + i];
  __syncthreads();
  const int nb = (n + 63) / 64;
  const int npairs = GGA ? nb * nb : nb * (nb + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
  for (int q = blockIdx.y; q < npairs; q += gridDim.y) {
    int I, J;
    pair_of(q, nb, GGA, I, J);
    Acc acc;
    acc.zero();
    // acc[j][i] = sum_p phi_j Z_i: rows of the fragment run along j, so the
    // atomics of a warp instruction hit 4 rows of V in runs of 8 functions
    gemm_tile<true, true>(acc, phi + sb * 128, 128, (int64_t)J * 64, Z + sb * 128, 128, (int64_t)I * 64, 0, 128,
                          smem);
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = J * 64 + wm0 + jj * 8 + (lane >> 2);
      const int fj = j < n ? sfn[j] : -1;
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = I * 64 + wn0 + ii * 8 + 2 * (lane & 3) + e;
          const int fi = i < n ? sfn[i] : -1;
          if (fi >= 0 && fj >= 0 && (GGA || fj >= fi)) atomicAdd(V + (int64_t)fi * ldv + fj, acc.v[jj][ii][e]);
        }
    }
  }
}

}  // namespace

// ham[spin + ispin*(j(j+1)/2 + k)] = H(k, j), k <= j; GGA: H(k, j) + H(j, k)
__global__ void k_spack(const double* __restrict__ V, int64_t nbas, bool sym2, int ispin, int spin,
                        double* __restrict__ ham) {
  const int64_t len = nbas * (nbas + 1) / 2;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < len;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > idx) --j;
    while ((j + 1) * (j + 2) / 2 <= idx) ++j;
    const int64_t k = idx - j * (j + 1) / 2;
    double v = V[k * nbas + j];
    if (sym2) v += V[j * nbas + k];
    ham[spin + (int64_t)ispin * idx] = v;
  }
}

// ---------------------------------------------------------------------------
// host planning
// ---------------------------------------------------------------------------
namespace {

// Squared radius beyond which radial function rr of shell S is dropped.
double listing_r2(const DevShell& S, int rr, const double* exps, const double* norms, const double* contr,
                  double threshold, double sa_fac) {
  std::vector<double> cf((size_t)S.nexp, 0.0);
  if (rr < S.nunc) cf[(size_t)rr] = 1.0;
  else
    for (int e = 0; e < S.nexp; ++e) cf[(size_t)e] = contr[S.con_off + e + (int64_t)S.nexp * (rr - S.nunc)];
  double amin = 1e300;
  for (int e = 0; e < S.nexp; ++e)
    if (cf[(size_t)e] != 0.0) amin = std::min(amin, exps[S.exp_off + e]);
  if (amin == 1e300) return 0.0;  // identically zero function
  // every primitive vanishes where alpha_min r^2 >= 50; margin for rounding
  const double r2cut = 50.0 / amin * (1.0 + 1e-9);
  if (threshold <= 0.0) return r2cut;
  // bound on |phi| and |grad phi| at distance r:
  //   sum_e |c_e| N_e exp(-a_e r^2) (r^l + 2 a_e r^(l+1) + (2l+1) r^(l-1)) * sa_fac
  const int l = S.l;
  auto bound = [&](double r) {
    double b = 0.0;
    for (int e = 0; e < S.nexp; ++e) {
      if (cf[(size_t)e] == 0.0) continue;
      const double a = exps[S.exp_off + e];
      if (a * r * r >= 50.0) continue;
      const double g = std::fabs(cf[(size_t)e]) * norms[S.exp_off + e] * std::exp(-a * r * r);
      double poly = std::pow(r, l) + 2.0 * a * std::pow(r, l + 1);
      if (l > 0) poly += (2 * l + 1) * std::pow(r, l - 1);
      b += g * poly;
    }
    return b * sa_fac;
  };
  const double rcut = std::sqrt(r2cut);
  const int nstep = 4000;
  const double dr = rcut / nstep;
  for (int i = nstep; i >= 0; --i) {
    const double r = i * dr;
    if (bound(r) >= threshold) {
      const double R = std::min(rcut, r + dr);
      return R * R;
    }
  }
  return 0.0;
}

}  // namespace

void screen_destroy(ScreenPlan* sp) {
  if (!sp) return;
  if (sp->mixed) screen_mixed_destroy(sp->mixed);
  for (void* p : sp->allocs) cudaFree(p);
  for (auto& e : sp->ev)
    if (e) cudaEventDestroy(e);
  delete sp;
}

void screen_stats(const ScreenPlan* sp, int64_t* ntiles, int64_t* nslots, int64_t* nlisted, double* sum_n2,
                  int64_t* nchunks) {
  if (ntiles) *ntiles = sp->ntiles;
  if (nslots) *nslots = sp->nslots;
  if (nlisted) *nlisted = sp->nlisted;
  if (sum_n2) *sum_n2 = sp->sum_n2;
  if (nchunks) *nchunks = (int64_t)sp->chunk_t0.size() - 1;
}

#define SP_TRY(call, what)                                                       \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      err = std::string(what) + ": " + cudaGetErrorString(e_);                   \
      screen_destroy(sp);                                                        \
      return e_ == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA;         \
    }                                                                            \
  } while (0)

int screen_create(ScreenPlan** out, const ScreenInput& in, const BuildArgs& a, cudaStream_t st, std::string& err) {
  *out = nullptr;
  ScreenPlan* sp = new ScreenPlan();
  sp->gga = in.gga;
  sp->mgga = in.mgga;
  sp->functional = in.functional;
  // The INT8 build keeps grad phi in FP32 (phi stays FP64): its density
  // gradient and potential then move 12 fewer bytes per basis value, within
  // the mixed-mode bars (measured on CH60-PBE: |dE_xc| 9.7e-8 Eh, max |dV_xc|
  // 3.1e-8 against the FP64 build; FP32 phi too would give 1.1e-6 Eh).  The
  // meta-GGA tau contractions run on the FP64 kernels and keep FP64 gradients.
  sp->gf32 = in.precision != PGXC_PREC_FP64 && in.gga && !in.mgga;
  sp->ispin = in.ispin;
  sp->nbas = in.nbas;
  sp->keep = in.keep_basis;
  const std::vector<DevShell>& shells = *in.shells;
  for (const DevShell& S : shells) {
    sp->n_exps = std::max<int64_t>(sp->n_exps, S.exp_off + S.nexp);
    sp->n_contr = std::max<int64_t>(sp->n_contr, S.con_off + (int64_t)S.nexp * S.ncontr);
    if (S.seg) sp->n_rng = std::max<int64_t>(sp->n_rng, S.rad_off + S.ncontr);
  }
  for (const DevShell& S : shells)
    if (S.nrad > 64) {
      err = "screened build: a shell has more than 64 radial functions";
      screen_destroy(sp);
      return PGXC_ENOTSUP;
    }
  for (auto& e : sp->ev) SP_TRY(cudaEventCreate(&e), "cudaEventCreate");
  {
    int dev = 0;
    SP_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    SP_TRY(cudaDeviceGetAttribute(&sp->nsm, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  }
  // --- Morton-ordered, 128-point tiles -----------------------------------
  const int64_t n = in.npts;
  const int64_t ntiles = (n + 127) / 128;
  sp->ntiles = ntiles;
  {
    // Morton order of the points, on the device (ties by point index)
    const int64_t nq = ntiles * 128;
    int64_t* dperm;
    SP_TRY(cudaMalloc(&dperm, sizeof(int64_t) * nq), "cudaMalloc");
    cudaError_t e = morton_perm_device(a.px, a.py, a.pz, n, nq, dperm, st);
    if (e == cudaSuccess) e = sp_alloc(sp, &sp->qx, 4 * nq);
    if (e == cudaSuccess) {
      sp->qy = sp->qx + nq;
      sp->qz = sp->qx + 2 * nq;
      sp->qw = sp->qx + 3 * nq;
      k_gather_points<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(dperm, nq, a.px, a.py, a.pz, a.w, sp->qx,
                                                                   sp->qy, sp->qz, sp->qw);
      e = cudaStreamSynchronize(st);
    }
    cudaFree(dperm);
    SP_TRY(e, "grid reordering");
  }
  // --- tile-atom distances ------------------------------------------------
  std::vector<float> d2((size_t)ntiles * in.natm);
  {
    float* dd2;
    SP_TRY(cudaMalloc(&dd2, sizeof(float) * d2.size()), "cudaMalloc");
    k_tile_atom_d2<<<(unsigned)ntiles, 128, 0, st>>>(sp->qx, sp->qy, sp->qz, a.atoms, in.natm, dd2);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaMemcpy(d2.data(), dd2, sizeof(float) * d2.size(), cudaMemcpyDeviceToHost);
    cudaFree(dd2);
    SP_TRY(e, "tile distances");
  }
  // --- listing radii -------------------------------------------------------
  double sa_fac[kMaxL + 1];
  for (int l = 0; l <= kMaxL; ++l) {
    sa_fac[l] = 1.0;
    if (!a.sa.identity)
      for (int i = 0; i < 2 * l + 1; ++i) {
        double s = 0.0;
        for (int m = 0; m < 2 * l + 1; ++m) s += std::fabs(a.sa.c[l][i][m]);
        sa_fac[l] = std::max(sa_fac[l], s);
      }
  }
  const int nsh = (int)shells.size();
  std::vector<std::vector<double>> R2((size_t)nsh);
  std::vector<double> shR2((size_t)nsh, 0.0);
  for (int s = 0; s < nsh; ++s) {
    const DevShell& S = shells[(size_t)s];
    R2[(size_t)s].resize((size_t)S.nrad);
    for (int rr = 0; rr < S.nrad; ++rr) {
      R2[(size_t)s][(size_t)rr] = listing_r2(S, rr, in.exps, in.norms, in.contr, in.threshold, sa_fac[S.l]);
      shR2[(size_t)s] = std::max(shR2[(size_t)s], R2[(size_t)s][(size_t)rr]);
    }
  }
  // --- per-tile lists --------------------------------------------------------
  std::vector<int64_t> tso((size_t)ntiles + 1, 0);
  std::vector<int> slot_fn, slot_tile, listed_t((size_t)ntiles, 0);
  std::vector<BasisItem> items[kMaxL + 1];
  std::vector<int64_t> tile_items[kMaxL + 1];  // items before tile t, per L
  for (int l = 0; l <= kMaxL; ++l) tile_items[l].assign((size_t)ntiles + 1, 0);
  slot_fn.reserve((size_t)ntiles * 64);
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t base = (int64_t)slot_fn.size();
    for (int l = 0; l <= kMaxL; ++l) tile_items[l][(size_t)t] = (int64_t)items[l].size();
    for (int s = 0; s < nsh; ++s) {
      const DevShell& S = shells[(size_t)s];
      const double dd = d2[(size_t)t * in.natm + S.atom];
      if (!(dd < shR2[(size_t)s])) continue;
      uint64_t mask = 0;
      for (int rr = 0; rr < S.nrad; ++rr)
        if (dd < R2[(size_t)s][(size_t)rr]) mask |= 1ull << rr;
      const int nsig = __builtin_popcountll(mask);
      BasisItem it{};
      it.ax = in.atoms[3 * S.atom];
      it.ay = in.atoms[3 * S.atom + 1];
      it.az = in.atoms[3 * S.atom + 2];
      it.tile = (int)t;
      it.slot = (int64_t)slot_fn.size();
      it.nsig = nsig;
      it.mask = mask;
      it.exp_off = S.exp_off;
      it.con_off = S.con_off;
      it.rad_off = S.rad_off;
      it.nexp = S.nexp;
      it.nunc = S.nunc;
      it.seg = S.seg;
      items[S.l].push_back(it);
      for (int i = 0; i < 2 * S.l + 1; ++i)
        for (int rr = 0; rr < S.nrad; ++rr)
          if (mask >> rr & 1) slot_fn.push_back(S.f0 + i * S.nrad + rr);
    }
    const int64_t listed = (int64_t)slot_fn.size() - base;
    listed_t[(size_t)t] = (int)listed;
    sp->nlisted += listed;
    while (((int64_t)slot_fn.size() - base) % kSlotAlign) slot_fn.push_back(-1);
    const int64_t nt = (int64_t)slot_fn.size() - base;
    sp->sum_n2 += (double)listed * (double)listed;
    sp->max_n = std::max(sp->max_n, (int)nt);
    slot_tile.resize(slot_fn.size(), (int)t);
    tso[(size_t)t + 1] = (int64_t)slot_fn.size();
  }
  for (int l = 0; l <= kMaxL; ++l) {
    tile_items[l][(size_t)ntiles] = (int64_t)items[l].size();
    sp->tile_item[l] = tile_items[l];
  }
  sp->nslots = (int64_t)slot_fn.size();
  sp->h_tso = tso;
  // --- chunks -------------------------------------------------------------------
  const bool mixed = in.precision != PGXC_PREC_FP64;
  size_t freeb = 0, totb = 0;
  SP_TRY(cudaMemGetInfo(&freeb, &totb), "cudaMemGetInfo");
  if (sp->keep) {
    // resident basis values and point digits of every slot: phi (+ grad phi), INT8 digits
    const double gb = in.gga ? 3.0 * (sp->gf32 ? 4.0 : 8.0) : 0.0;
    const double need = (double)(sp->nslots + kSlack) * 128 * (8.0 + gb + (mixed ? 5.0 : 0.0));
    if (need > 0.6 * (double)freeb) {
      err = "screened build: the basis values of the whole grid (" + std::to_string((int64_t)(need / 1e9)) +
            " GB) do not fit beside the build's buffers; create the context without keep_orbitals";
      screen_destroy(sp);
      return PGXC_ENOMEM;
    }
    freeb -= (size_t)need;
  }
  const int64_t per_slot = 128 * (16 + (in.gga ? 3 * (sp->gf32 ? 4 : 8) : 0)) + (mixed ? screen_mixed_bytes_per_slot() : 0);
  const int64_t per_tile = 128 * 8 * 8 * in.ispin + (mixed ? screen_mixed_bytes_per_tile() : 0);
  int64_t budget_slots = (int64_t)(0.45 * (double)freeb) / per_slot;
  budget_slots = std::max<int64_t>(budget_slots, sp->max_n);
  int64_t budget_tiles = std::max<int64_t>(1, (int64_t)(0.05 * (double)freeb) / per_tile);
  if (in.max_chunk_points > 0) budget_tiles = std::min(budget_tiles, std::max<int64_t>(1, in.max_chunk_points / 128));
  budget_tiles = std::min<int64_t>(budget_tiles, 1 << 16);
  // INT8 path: the gathered density B operand, per tile
  std::vector<int64_t> boff((size_t)ntiles + 1, 0);
  if (mixed)
    for (int64_t t = 0; t < ntiles; ++t)
      boff[(size_t)t + 1] = boff[(size_t)t] + screen_mixed_bstages(tso[(size_t)t + 1] - tso[(size_t)t]);
  const int64_t budget_bstages =
      mixed ? std::max<int64_t>((int64_t)(0.25 * (double)freeb) / screen_mixed_bytes_per_bstage(),
                                screen_mixed_bstages(sp->max_n))
            : INT64_MAX;
  sp->chunk_t0.push_back(0);
  {
    int64_t t0 = 0;
    for (int64_t t = 0; t < ntiles; ++t) {
      const bool full_slots = tso[(size_t)t + 1] - tso[(size_t)t0] > budget_slots;
      const bool full_tiles = t - t0 + 1 > budget_tiles;
      const bool full_b = boff[(size_t)t + 1] - boff[(size_t)t0] > budget_bstages;
      if (t > t0 && (full_slots || full_tiles || full_b)) {
        sp->chunk_t0.push_back(t);
        t0 = t;
      }
    }
    sp->chunk_t0.push_back(ntiles);
  }
  int64_t chunk_bstages = 0;
  const size_t nch = sp->chunk_t0.size() - 1;
  for (size_t c = 0; c < nch; ++c) {
    const int64_t t0 = sp->chunk_t0[c], t1 = sp->chunk_t0[c + 1];
    sp->chunk_tiles = std::max(sp->chunk_tiles, t1 - t0);
    sp->chunk_slots = std::max(sp->chunk_slots, tso[(size_t)t1] - tso[(size_t)t0]);
    chunk_bstages = std::max(chunk_bstages, boff[(size_t)t1] - boff[(size_t)t0]);
  }
  for (int l = 0; l <= kMaxL; ++l)
    for (size_t c = 0; c <= nch; ++c) sp->item_off[l].push_back(tile_items[l][(size_t)sp->chunk_t0[c]]);
  // --- device copies and buffers ------------------------------------------------
  SP_TRY(sp_alloc(sp, &sp->tso, tso.size()), "cudaMalloc");
  SP_TRY(cudaMemcpy(sp->tso, tso.data(), sizeof(int64_t) * tso.size(), cudaMemcpyHostToDevice), "copy");
  SP_TRY(sp_alloc(sp, &sp->listed, listed_t.size()), "cudaMalloc");
  SP_TRY(cudaMemcpy(sp->listed, listed_t.data(), sizeof(int) * listed_t.size(), cudaMemcpyHostToDevice), "copy");
  SP_TRY(sp_alloc(sp, &sp->slot_fn, slot_fn.size()), "cudaMalloc");
  SP_TRY(sp_alloc(sp, &sp->slot_tile, slot_tile.size()), "cudaMalloc");
  if (!slot_fn.empty()) {
    SP_TRY(cudaMemcpy(sp->slot_fn, slot_fn.data(), sizeof(int) * slot_fn.size(), cudaMemcpyHostToDevice), "copy");
    SP_TRY(cudaMemcpy(sp->slot_tile, slot_tile.data(), sizeof(int) * slot_tile.size(), cudaMemcpyHostToDevice),
           "copy");
  }
  for (int l = 0; l <= kMaxL; ++l) {
    SP_TRY(sp_alloc(sp, &sp->items[l], items[l].size()), "cudaMalloc");
    if (!items[l].empty())
      SP_TRY(cudaMemcpy(sp->items[l], items[l].data(), sizeof(BasisItem) * items[l].size(), cudaMemcpyHostToDevice),
             "copy");
  }
  const size_t rows = (size_t)(sp->chunk_slots + kSlack) * 128;
  // basis arrays: one chunk's rows, or every slot of the grid when they stay resident
  const size_t brows = sp->keep ? (size_t)(sp->nslots + kSlack) * 128 : rows;
  SP_TRY(sp_alloc(sp, &sp->phi, brows), "cudaMalloc (phi)");
  SP_TRY(sp_alloc(sp, &sp->Z, rows), "cudaMalloc (Z)");
  SP_TRY(cudaMemset(sp->phi, 0, sizeof(double) * brows), "memset");
  SP_TRY(cudaMemset(sp->Z, 0, sizeof(double) * rows), "memset");
  if (in.gga && sp->gf32) {
    SP_TRY(sp_alloc(sp, &sp->fx, brows), "cudaMalloc (grad phi)");
    SP_TRY(sp_alloc(sp, &sp->fy, brows), "cudaMalloc (grad phi)");
    SP_TRY(sp_alloc(sp, &sp->fz, brows), "cudaMalloc (grad phi)");
    SP_TRY(cudaMemset(sp->fx, 0, sizeof(float) * brows), "memset");
    SP_TRY(cudaMemset(sp->fy, 0, sizeof(float) * brows), "memset");
    SP_TRY(cudaMemset(sp->fz, 0, sizeof(float) * brows), "memset");
  } else if (in.gga) {
    SP_TRY(sp_alloc(sp, &sp->gx, brows), "cudaMalloc (grad phi)");
    SP_TRY(sp_alloc(sp, &sp->gy, brows), "cudaMalloc (grad phi)");
    SP_TRY(sp_alloc(sp, &sp->gz, brows), "cudaMalloc (grad phi)");
    SP_TRY(cudaMemset(sp->gx, 0, sizeof(double) * brows), "memset");
    SP_TRY(cudaMemset(sp->gy, 0, sizeof(double) * brows), "memset");
    SP_TRY(cudaMemset(sp->gz, 0, sizeof(double) * brows), "memset");
  }
  const int64_t cp = sp->chunk_tiles * 128;
  SP_TRY(sp_alloc(sp, &sp->pt, 8 * (size_t)in.ispin * cp), "cudaMalloc");
  SP_TRY(cudaMemset(sp->pt, 0, sizeof(double) * 8 * in.ispin * cp), "memset");
  if (in.mgga) {
    SP_TRY(sp_alloc(sp, &sp->tq, 4 * (size_t)in.ispin * cp), "cudaMalloc");
    SP_TRY(cudaMemset(sp->tq, 0, sizeof(double) * 4 * in.ispin * cp), "memset");
  }
  SP_TRY(sp_alloc(sp, &sp->partial, 2 * (size_t)((cp + 255) / 256) + 2), "cudaMalloc");
  SP_TRY(sp_alloc(sp, &sp->V, (size_t)in.ispin * in.nbas * in.nbas), "cudaMalloc (V)");
  if (mixed) {
    ScreenMixedInput mi;
    mi.nbas = in.nbas;
    mi.ldc = a.ldc;
    mi.gga = in.gga;
    mi.nspin = in.ispin;
    mi.chunk_slots = sp->chunk_slots + kSlack;
    mi.chunk_tiles = sp->chunk_tiles;
    mi.max_n = sp->max_n;
    mi.chunk_bstages = chunk_bstages;
    if (sp->keep) {
      mi.resident_slots = sp->nslots + kSlack;
      mi.resident_tiles = sp->ntiles;
    }
    SP_TRY(sp_alloc(sp, &sp->pmax, (size_t)sp->chunk_tiles * 128), "cudaMalloc");
    SP_TRY(sp_alloc(sp, &sp->b_off, boff.size()), "cudaMalloc");
    SP_TRY(cudaMemcpy(sp->b_off, boff.data(), sizeof(int64_t) * boff.size(), cudaMemcpyHostToDevice), "copy");
    mi.b_off = sp->b_off;
    const int st2 = screen_mixed_create(&sp->mixed, mi, err);
    if (st2) {
      screen_destroy(sp);
      return st2;
    }
  }
  *out = sp;
  return PGXC_OK;
}

int screen_run(ScreenPlan* sp, const BuildArgs& a, const double* Pb, cudaStream_t st, double* ham, ScreenTimes* tm,
               std::string& err, const ScreenExtra* extra) {
  const bool potential = !extra || extra->potential;
  const bool gga = sp->gga;
  const int ispin = sp->ispin;
  const double* P[2] = {a.P, Pb};
  const int64_t nb2 = sp->nbas * sp->nbas;
  const bool timed = tm != nullptr;  // untimed: no event records, synchronisation or host reads (capturable)
  // resident basis values filled by an earlier build: skip their evaluation (K1)
  const bool eval_basis = !(sp->keep && sp->basis_ready);
  ScreenTimes T;
  cudaEvent_t* ev = sp->ev;
#define SR_TRY(call)                                                          \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      err = std::string("screened build: ") + cudaGetErrorString(e_);         \
      return PGXC_ECUDA;                                                      \
    }                                                                         \
  } while (0)
  SR_TRY(cudaMemsetAsync(sp->V, 0, sizeof(double) * ispin * nb2, st));
  if (sp->mixed) {
    if (timed) SR_TRY(cudaEventRecord(ev[0], st));
    for (int s = 0; s < ispin; ++s) T.launches += screen_mixed_prepare(sp->mixed, P[s], a.ldc, s, st);
    SR_TRY(cudaGetLastError());
    if (timed) SR_TRY(cudaEventRecord(ev[1], st));
  }
  const int64_t cp = sp->chunk_tiles * 128;
  // per-chunk point arrays of spin s: 8 columns of cp (rho, grad rho, A, B) from pt + 8 s cp
  BuildArgs b[2];
  for (int s = 0; s < ispin; ++s) {
    double* q = sp->pt + 8 * s * cp;
    b[s] = a;
    b[s].ldp = cp;
    b[s].w = nullptr;
    b[s].rho = q;
    b[s].grx = q + cp;
    b[s].gry = q + 2 * cp;
    b[s].grz = q + 3 * cp;
    b[s].A = q + 4 * cp;
    b[s].Bx = q + 5 * cp;
    b[s].By = q + 6 * cp;
    b[s].Bz = q + 7 * cp;
    b[s].partial = sp->partial;
  }
  const size_t nch = sp->chunk_t0.size() - 1;
  float ms;
  for (size_t c = 0; c < nch; ++c) {
    const int64_t t0 = sp->chunk_t0[c], t1 = sp->chunk_t0[c + 1], nt = t1 - t0;
    const int64_t s0 = sp->h_tso[(size_t)t0], ns = sp->h_tso[(size_t)t1] - s0;
    const int64_t npt = nt * 128;
    // this chunk's rows of the basis arrays (resident: the chunk's place among all slots)
    const int64_t so = sp->keep ? s0 : 0, to = sp->keep ? t0 : 0;
    double* phi = sp->phi + so * 128;
    const bool gf = sp->gf32;
    double* gxc = gga && !gf ? sp->gx + so * 128 : nullptr;
    double* gyc = gga && !gf ? sp->gy + so * 128 : nullptr;
    double* gzc = gga && !gf ? sp->gz + so * 128 : nullptr;
    float* fxc = gga && gf ? sp->fx + so * 128 : nullptr;
    float* fyc = gga && gf ? sp->fy + so * 128 : nullptr;
    float* fzc = gga && gf ? sp->fz + so * 128 : nullptr;
    if (timed) SR_TRY(cudaEventRecord(ev[2], st));
    // K1
    if (!eval_basis) {
      if (sp->mixed) T.launches += screen_mixed_gather(sp->mixed, sp->tso, sp->slot_fn, t0, nt, s0, 0, st);
    } else {
      if (sp->pmax) SR_TRY(cudaMemsetAsync(sp->pmax, 0, sizeof(unsigned long long) * nt * 128, st));
      auto launch_l = [&](auto Lc) {
        constexpr int L = decltype(Lc)::value;
        const int64_t i0 = sp->item_off[L][c], i1 = sp->item_off[L][c + 1];
        if (i1 <= i0) return;
        // persistent-style blocks, each walking a contiguous range of items
        const unsigned nb = (unsigned)std::min<int64_t>(i1 - i0, (int64_t)sp->nsm * kBasisBlocksPerSM);
        if (gga && gf)
          k_basis_items<L, true, float><<<nb, 128, 0, st>>>(sp->items[L] + i0, i1 - i0, a.exps, a.norms, a.contr,
                                                            a.rng, a.sa, sp->qx, sp->qy, sp->qz, s0, t0, phi, fxc, fyc,
                                                            fzc, sp->pmax);
        else if (gga)
          k_basis_items<L, true><<<nb, 128, 0, st>>>(sp->items[L] + i0, i1 - i0, a.exps, a.norms, a.contr, a.rng,
                                                     a.sa, sp->qx, sp->qy, sp->qz, s0, t0, phi, gxc, gyc, gzc, sp->pmax);
        else
          k_basis_items<L, false, double><<<nb, 128, 0, st>>>(sp->items[L] + i0, i1 - i0, a.exps, a.norms, a.contr,
                                                              a.rng, a.sa, sp->qx, sp->qy, sp->qz, s0, t0, phi,
                                                              (double*)nullptr, (double*)nullptr, (double*)nullptr,
                                                              sp->pmax);
        ++T.launches;
      };
      launch_l(std::integral_constant<int, 0>());
      launch_l(std::integral_constant<int, 1>());
      launch_l(std::integral_constant<int, 2>());
      launch_l(std::integral_constant<int, 3>());
      if (gga && gf) k_pad_zero<true, float><<<(unsigned)nt, 128, 0, st>>>(sp->tso, sp->listed, t0, s0, phi, fxc, fyc, fzc);
      else if (gga) k_pad_zero<true><<<(unsigned)nt, 128, 0, st>>>(sp->tso, sp->listed, t0, s0, phi, gxc, gyc, gzc);
      else k_pad_zero<false, double><<<(unsigned)nt, 128, 0, st>>>(sp->tso, sp->listed, t0, s0, phi, (double*)nullptr,
                                                                   (double*)nullptr, (double*)nullptr);
      ++T.launches;
      if (sp->mixed)
        T.launches += screen_mixed_basis(sp->mixed, sp->tso, sp->slot_fn, t0, nt, s0, phi, sp->pmax, so, to, st);
    }
    if (timed) SR_TRY(cudaEventRecord(ev[3], st));
    // K3, per spin
    if (timed) SR_TRY(cudaEventRecord(ev[4], st));
    for (int s = 0; s < ispin; ++s) {
      if (sp->mixed) {
        if (s > 0) T.launches += screen_mixed_gather(sp->mixed, sp->tso, sp->slot_fn, t0, nt, s0, s, st);
        if (gf)
          T.launches += screen_mixed_density(sp->mixed, sp->tso, sp->slot_fn, t0, nt, s0, phi, fxc, fyc, fzc,
                                             b[s].rho, b[s].grx, b[s].gry, b[s].grz, so, to, st);
        else
          T.launches += screen_mixed_density(sp->mixed, sp->tso, sp->slot_fn, t0, nt, s0, phi, gxc, gyc, gzc,
                                             b[s].rho, b[s].grx, b[s].gry, b[s].grz, so, to, st);
      } else {
        const int smem = gemm_smem_bytes<false, false>() + (int)sizeof(int) * sp->max_n;
        dim3 grid((unsigned)nt, 2);
        if (gga) {
          raise_smem_limit(k_sdensity<true>, smem);
          k_sdensity<true><<<grid, kGemmThreads, smem, st>>>(phi, gxc, gyc, gzc, sp->tso, t0, s0,
                                                             sp->slot_fn, P[s], a.ldc, b[s].rho, b[s].grx, b[s].gry,
                                                             b[s].grz);
        } else {
          raise_smem_limit(k_sdensity<false>, smem);
          k_sdensity<false><<<grid, kGemmThreads, smem, st>>>(phi, nullptr, nullptr, nullptr, sp->tso, t0, s0,
                                                              sp->slot_fn, P[s], a.ldc, b[s].rho, nullptr, nullptr,
                                                              nullptr);
        }
        ++T.launches;
      }
      if (sp->mgga || (extra && extra->tau)) {
        // 2 tau_j = sum_nu (d_j phi P)_nu d_j phi_nu: the density contraction with d_j phi in the
        // place of phi (FP64 DMMA in every precision mode)
        const int smem = gemm_smem_bytes<false, false>() + (int)sizeof(int) * sp->max_n;
        raise_smem_limit(k_sdensity<false>, smem);
        const double* gj[3] = {gxc, gyc, gzc};
        for (int j = 0; j < 3; ++j) {
          k_sdensity<false><<<dim3((unsigned)nt, 2), kGemmThreads, smem, st>>>(
              gj[j], nullptr, nullptr, nullptr, sp->tso, t0, s0, sp->slot_fn, P[s], a.ldc,
              sp->tq + (4 * s + j) * cp, nullptr, nullptr, nullptr);
          ++T.launches;
        }
      }
    }
    if (timed) SR_TRY(cudaEventRecord(ev[5], st));
    // K2
    if (sp->mgga) {
      launch_functional_mgga(sp->functional, ispin, sp->qw, sp->pt, sp->tq, cp, t0 * 128, npt, sp->partial, a.acc,
                             st);
    } else if (ispin == 1) {
      BuildArgs bf = b[0];
      bf.w = sp->qw;
      launch_functional_f64(bf, t0 * 128, npt, gga, st);
    } else {
      launch_functional2_f64(a.xc, sp->qw, b[0].rho, b[1].rho, cp, t0 * 128, npt, gga, sp->partial, a.acc, st);
    }
    T.launches += 2;
    if (timed) SR_TRY(cudaEventRecord(ev[6], st));
    // K4, per spin: the contraction of spin s is bracketed by ev[7 + 3s], ev[8 + 3s]
    for (int s = 0; s < ispin && potential; ++s) {
      double* Vs = sp->V + s * nb2;
      cudaEvent_t k0 = timed ? ev[7 + 3 * s] : nullptr, k1 = timed ? ev[8 + 3 * s] : nullptr;
      if (sp->mixed) {
        if (gf)
          T.launches += screen_mixed_potential(sp->mixed, sp->tso, sp->slot_fn, sp->slot_tile, t0, nt, s0, ns, phi,
                                               fxc, fyc, fzc, b[s].A, b[s].Bx, b[s].By, b[s].Bz, Vs, sp->nbas,
                                               st, k0, k1);
        else
          T.launches += screen_mixed_potential(sp->mixed, sp->tso, sp->slot_fn, sp->slot_tile, t0, nt, s0, ns, phi,
                                               gxc, gyc, gzc, b[s].A, b[s].Bx, b[s].By, b[s].Bz, Vs, sp->nbas,
                                               st, k0, k1);
      } else {
        const unsigned nbk = (unsigned)std::max<int64_t>(1, std::min<int64_t>((ns * 128 + 255) / 256, 148 * 32));
        if (gga)
          k_szbuild<true><<<nbk, 256, 0, st>>>(ns, sp->slot_tile + s0, t0, phi, gxc, gyc, gzc, b[s].A,
                                               b[s].Bx, b[s].By, b[s].Bz, sp->Z);
        else
          k_szbuild<false><<<nbk, 256, 0, st>>>(ns, sp->slot_tile + s0, t0, phi, nullptr, nullptr, nullptr,
                                                b[s].A, nullptr, nullptr, nullptr, sp->Z);
        if (timed) SR_TRY(cudaEventRecord(k0, st));
        const int smem = gemm_smem_bytes<true, true>() + (int)sizeof(int) * sp->max_n;
        dim3 grid((unsigned)nt, 4);
        if (gga) {
          raise_smem_limit(k_svpot<true>, smem);
          k_svpot<true><<<grid, kGemmThreads, smem, st>>>(phi, sp->Z, sp->tso, t0, s0, sp->slot_fn, Vs,
                                                          sp->nbas);
        } else {
          raise_smem_limit(k_svpot<false>, smem);
          k_svpot<false><<<grid, kGemmThreads, smem, st>>>(phi, sp->Z, sp->tso, t0, s0, sp->slot_fn, Vs,
                                                           sp->nbas);
        }
        if (timed) SR_TRY(cudaEventRecord(k1, st));
        T.launches += 2;
      }
      if (sp->mgga) {
        // tau term: per direction Z = C d_j phi and H += Z^T d_j phi over the whole square of
        // each tile (k_spack then forms H + H^T), FP64 DMMA in every precision mode
        const unsigned nbk = (unsigned)std::max<int64_t>(1, std::min<int64_t>((ns * 128 + 255) / 256, 148 * 32));
        const int smem = gemm_smem_bytes<true, true>() + (int)sizeof(int) * sp->max_n;
        raise_smem_limit(k_svpot<true>, smem);
        const double* gj[3] = {gxc, gyc, gzc};
        const double* Cs = sp->tq + (4 * s + 3) * cp;
        for (int j = 0; j < 3; ++j) {
          k_szbuild<false><<<nbk, 256, 0, st>>>(ns, sp->slot_tile + s0, t0, gj[j], nullptr, nullptr, nullptr, Cs,
                                                nullptr, nullptr, nullptr, sp->Z);
          k_svpot<true><<<dim3((unsigned)nt, 4), kGemmThreads, smem, st>>>(gj[j], sp->Z, sp->tso, t0, s0,
                                                                            sp->slot_fn, Vs, sp->nbas);
          T.launches += 2;
        }
      }
    }
    // further functionals on the same density (after K4, whose A and B they overwrite)
    for (int i = 0; extra && i < extra->n; ++i) {
      if (extra->fid && PGXC_XC_IS_MGGA(extra->fid[i])) {
        launch_functional_mgga(extra->fid[i], ispin, sp->qw, sp->pt, sp->tq, cp, t0 * 128, npt, sp->partial,
                               extra->acc + 4 * i, st);
      } else if (ispin == 1) {
        BuildArgs bx = b[0];
        bx.w = sp->qw;
        bx.xc = extra->xc[i];
        bx.acc = extra->acc + 4 * i;
        launch_functional_f64(bx, t0 * 128, npt, extra->gga[i] != 0, st);
      } else {
        launch_functional2_f64(extra->xc[i], sp->qw, b[0].rho, b[1].rho, cp, t0 * 128, npt, extra->gga[i] != 0,
                               sp->partial, extra->acc + 4 * i, st);
      }
      T.launches += 2;
    }
    SR_TRY(cudaGetLastError());
    if (!timed) continue;
    SR_TRY(cudaEventRecord(ev[9], st));
    SR_TRY(cudaEventSynchronize(ev[9]));
    SR_TRY(cudaEventElapsedTime(&ms, ev[2], ev[3])); T.basis += ms;
    SR_TRY(cudaEventElapsedTime(&ms, ev[4], ev[5])); T.density += ms; T.x += ms;
    SR_TRY(cudaEventElapsedTime(&ms, ev[5], ev[6])); T.functional += ms;
    SR_TRY(cudaEventElapsedTime(&ms, ev[6], ev[9])); T.potential += ms;
    for (int s = 0; s < ispin; ++s) {
      SR_TRY(cudaEventElapsedTime(&ms, ev[7 + 3 * s], ev[8 + 3 * s]));
      T.v += ms;
    }
  }
  if (sp->mixed && timed) {
    SR_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    T.density += ms;
  }
  if (timed) SR_TRY(cudaEventRecord(ev[2], st));
  if (potential) {
    const int64_t len = sp->nbas * (sp->nbas + 1) / 2;
    const unsigned nbk = (unsigned)std::min<int64_t>((len + 255) / 256, 148 * 8);
    for (int s = 0; s < ispin; ++s) {
      k_spack<<<nbk, 256, 0, st>>>(sp->V + s * nb2, sp->nbas, gga, ispin, s, ham);
      ++T.launches;
    }
  }
  SR_TRY(cudaGetLastError());
  if (!timed) return PGXC_OK;
  SR_TRY(cudaEventRecord(ev[3], st));
  SR_TRY(cudaEventSynchronize(ev[3]));
  SR_TRY(cudaEventElapsedTime(&ms, ev[2], ev[3]));
  T.potential += ms;
  if (sp->mixed) {
    int flag = 0;
    if (screen_mixed_error_flag(sp->mixed, st, &flag) != PGXC_OK) {
      err = "screened build: error-flag read failed";
      return PGXC_ECUDA;
    }
    if (flag) {
      err = "screened build: a bounded tensor-core pipeline wait ran out";
      return PGXC_ETIMEOUT;
    }
  }
#undef SR_TRY
  if (sp->keep) sp->basis_ready = true;  // a completed build has filled the resident basis values
  *tm = T;
  return PGXC_OK;
}

int screen_enable_tau(ScreenPlan* sp, std::string& err) {
  if (sp->tq) return PGXC_OK;
  if (!sp->gga || sp->gf32) {
    err = "meta-GGA energies need the FP64 gradient planes of a GGA (or a meta-GGA) context";
    return PGXC_ENOTSUP;
  }
  const int64_t cp = sp->chunk_tiles * 128;
  if (sp_alloc(sp, &sp->tq, 4 * (size_t)sp->ispin * cp) != cudaSuccess ||
      cudaMemset(sp->tq, 0, sizeof(double) * 4 * sp->ispin * cp) != cudaSuccess) {
    err = "meta-GGA energies: the tau buffer";
    return PGXC_ENOMEM;
  }
  return PGXC_OK;
}

int screen_error_flag(ScreenPlan* sp, cudaStream_t st, int* flag) {
  *flag = 0;
  if (!sp->mixed) return PGXC_OK;
  return screen_mixed_error_flag(sp->mixed, st, flag);
}


// ---------------------------------------------------------------------------
// Sets of contexts (screened.h): one launch per kernel over many contexts'
// tiles.
// ---------------------------------------------------------------------------
namespace {

// per context: where its E_xc / N_el accumulators, V and outputs live
struct SetOutDev {
  double* acc;        // {E, cE, N, cN}
  const double* V;    // [nbas][nbas]
  int64_t nbas;
  int gga;
  double* ham;        // packed out
  double* exc_nel;    // {E, N} out
};

// one segment of a chunk: tiles [t0, t0 + n) (chunk-relative) of context m
struct SetSeg {
  int64_t t0, n;
  int m;
  int pad_;
};

__global__ void k_set_adjust_items(BasisItem* __restrict__ it, int64_t n, int64_t dtile, int64_t dslot, int dexp,
                                   int dcon, int drng) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  it[i].tile += (int)dtile;
  it[i].slot += dslot;
  it[i].exp_off += dexp;
  it[i].con_off += dcon;
  it[i].rad_off += drng;
}

// Per segment (block): the fixed-order sum of its tiles' partials, Kahan-added
// into its context's acc.
__global__ void k_set_sum(const double* __restrict__ partial, const SetSeg* __restrict__ seg,
                          const SetOutDev* __restrict__ out) {
  const SetSeg g = seg[blockIdx.x];
  __shared__ double se[128], sq[128];
  double e = 0.0, q = 0.0;
  for (int64_t i = threadIdx.x; i < g.n; i += blockDim.x) {
    e += partial[2 * (g.t0 + i)];
    q += partial[2 * (g.t0 + i) + 1];
  }
  se[threadIdx.x] = e;
  sq[threadIdx.x] = q;
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sq[threadIdx.x] += sq[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* acc = out[g.m].acc;
    const double vals[2] = {se[0], sq[0]};
    for (int k = 0; k < 2; ++k) {
      const double y = vals[k] - acc[2 * k + 1];
      const double t = acc[2 * k] + y;
      acc[2 * k + 1] = (t - acc[2 * k]) - y;
      acc[2 * k] = t;
    }
  }
}

// Block per context: the packed triangle (tristore order; GGA: H + H^T) and
// {E_xc, N_el}.
__global__ void k_set_pack(const SetOutDev* __restrict__ out) {
  const SetOutDev o = out[blockIdx.x];
  const int64_t len = o.nbas * (o.nbas + 1) / 2;
  for (int64_t idx = threadIdx.x; idx < len; idx += blockDim.x) {
    int64_t j = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (j * (j + 1) / 2 > idx) --j;
    while ((j + 1) * (j + 2) / 2 <= idx) ++j;
    const int64_t k = idx - j * (j + 1) / 2;
    double v = o.V[k * o.nbas + j];
    if (o.gga) v += o.V[j * o.nbas + k];
    o.ham[idx] = v;
  }
  if (threadIdx.x == 0) {
    o.exc_nel[0] = o.acc[0];
    o.exc_nel[1] = o.acc[2];
  }
}

}  // namespace

struct ScreenSet {
  struct Group {
    XcConst xc;
    bool gga;
  };
  struct Chunk {
    int64_t t0, t1, s0;
    int64_t i0[kMaxL + 1], i1[kMaxL + 1];
    int group;
    int64_t seg0, nseg;
  };
  std::vector<SetMember> mem;
  std::vector<Group> groups;
  std::vector<Chunk> chunks;
  int64_t ntiles = 0, nslots = 0, chunk_slots = 0, chunk_tiles = 0;
  int max_n = 0;
  DevSA sa;
  // merged plan (device)
  double *qx = nullptr, *qy = nullptr, *qz = nullptr, *qw = nullptr;
  int64_t* tso = nullptr;
  int* slot_fn = nullptr;
  int* listed = nullptr;
  int* tile_mol = nullptr;
  BasisItem* items[kMaxL + 1] = {};
  double *exps = nullptr, *norms = nullptr, *contr = nullptr;
  int2* rng = nullptr;
  SetMolDev* mols = nullptr;
  SetOutDev* outs = nullptr;
  SetSeg* segs = nullptr;
  int64_t* b_off = nullptr;
  // chunk buffers
  double* phi = nullptr;
  float *gx = nullptr, *gy = nullptr, *gz = nullptr;  // grad phi in 32 bits (the INT8 build's)
  double* pt = nullptr;
  double* partial = nullptr;
  unsigned long long* pmax = nullptr;
  ScreenMixed* mixed = nullptr;
  int nsm = 148;
  int64_t launches = 0;
  std::vector<void*> allocs;
};

void screen_set_destroy(ScreenSet* s) {
  if (!s) return;
  if (s->mixed) screen_mixed_destroy(s->mixed);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

void screen_set_stats(const ScreenSet* s, int64_t* ntiles, int64_t* nchunks, int64_t* launches) {
  if (ntiles) *ntiles = s->ntiles;
  if (nchunks) *nchunks = (int64_t)s->chunks.size();
  if (launches) *launches = s->launches;
}

int screen_set_create(ScreenSet** out, const std::vector<SetMember>& members, int64_t max_chunk_points,
                      cudaStream_t st, std::string& err) {
  *out = nullptr;
  ScreenSet* S = new ScreenSet();
  auto fail = [&](int code, const std::string& m) {
    err = "set: " + m;
    screen_set_destroy(S);
    return code;
  };
#define SS_TRY(call, what)                                                                         \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(e_ == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA,                       \
                  std::string(what) + ": " + cudaGetErrorString(e_));                              \
  } while (0)
  auto alloc = [&](auto** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(**p));
    if (e == cudaSuccess) {
      S->allocs.push_back(q);
      *p = static_cast<std::remove_reference_t<decltype(*p)>>(q);
    }
    return e;
  };
  if (members.empty()) return fail(PGXC_EINVAL, "no contexts");
  // members grouped by functional (stable): a chunk holds one functional
  std::vector<int> order(members.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return members[(size_t)x].functional < members[(size_t)y].functional; });
  for (int i : order) S->mem.push_back(members[(size_t)i]);
  S->sa = S->mem[0].a->sa;
  for (const SetMember& m : S->mem) {
    const ScreenPlan* sp = m.sp;
    if (!sp->mixed || sp->ispin != 1 || sp->keep)
      return fail(PGXC_ENOTSUP, "every context must be a screened INT8 closed-shell one without keep_orbitals");
    if (!m.a->sa.identity) return fail(PGXC_ENOTSUP, "contexts with a symmetry adaptation table");
  }
  std::vector<int> mgroup(S->mem.size());
  for (size_t i = 0; i < S->mem.size(); ++i) {
    if (i == 0 || S->mem[i].functional != S->mem[i - 1].functional)
      S->groups.push_back({S->mem[i].a->xc, S->mem[i].sp->gga});
    mgroup[i] = (int)S->groups.size() - 1;
  }
  {
    int dev = 0;
    SS_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    SS_TRY(cudaDeviceGetAttribute(&S->nsm, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  }
  // --- merged plan -----------------------------------------------------------
  const size_t nm = S->mem.size();
  std::vector<int64_t> toff(nm + 1, 0), soff(nm + 1, 0), eoff(nm + 1, 0), coff(nm + 1, 0), roff(nm + 1, 0);
  std::vector<int64_t> ioff[kMaxL + 1];
  for (int l = 0; l <= kMaxL; ++l) ioff[l].assign(nm + 1, 0);
  for (size_t i = 0; i < nm; ++i) {
    const ScreenPlan* sp = S->mem[i].sp;
    toff[i + 1] = toff[i] + sp->ntiles;
    soff[i + 1] = soff[i] + sp->nslots;
    eoff[i + 1] = eoff[i] + sp->n_exps;
    coff[i + 1] = coff[i] + sp->n_contr;
    roff[i + 1] = roff[i] + sp->n_rng;
    for (int l = 0; l <= kMaxL; ++l) ioff[l][i + 1] = ioff[l][i] + sp->item_off[l].back();
    S->max_n = std::max(S->max_n, sp->max_n);
  }
  S->ntiles = toff[nm];
  S->nslots = soff[nm];
  const int64_t T = S->ntiles;
  SS_TRY(alloc(&S->qx, 4 * (size_t)T * 128), "cudaMalloc");
  S->qy = S->qx + T * 128;
  S->qz = S->qx + 2 * T * 128;
  S->qw = S->qx + 3 * T * 128;
  SS_TRY(alloc(&S->tso, (size_t)T + 1), "cudaMalloc");
  SS_TRY(alloc(&S->slot_fn, (size_t)S->nslots), "cudaMalloc");
  SS_TRY(alloc(&S->listed, (size_t)T), "cudaMalloc");
  SS_TRY(alloc(&S->tile_mol, (size_t)T), "cudaMalloc");
  SS_TRY(alloc(&S->exps, (size_t)eoff[nm]), "cudaMalloc");
  SS_TRY(alloc(&S->norms, (size_t)eoff[nm]), "cudaMalloc");
  SS_TRY(alloc(&S->contr, (size_t)coff[nm]), "cudaMalloc");
  SS_TRY(alloc(&S->rng, (size_t)roff[nm]), "cudaMalloc");
  for (int l = 0; l <= kMaxL; ++l) SS_TRY(alloc(&S->items[l], (size_t)ioff[l][nm]), "cudaMalloc");
  std::vector<int64_t> h_tso((size_t)T + 1, 0);
  std::vector<int> h_tile_mol((size_t)T);
  std::vector<SetMolDev> h_mols(nm);
  std::vector<SetOutDev> h_outs(nm);
  for (size_t i = 0; i < nm; ++i) {
    const ScreenPlan* sp = S->mem[i].sp;
    const BuildArgs* a = S->mem[i].a;
    const int64_t nt = sp->ntiles, t0 = toff[i];
    for (int c = 0; c < 4; ++c) {
      const double* src = c == 0 ? sp->qx : (c == 1 ? sp->qy : (c == 2 ? sp->qz : sp->qw));
      SS_TRY(cudaMemcpyAsync(S->qx + c * T * 128 + t0 * 128, src, sizeof(double) * nt * 128,
                             cudaMemcpyDeviceToDevice, st), "copy");
    }
    SS_TRY(cudaMemcpyAsync(S->slot_fn + soff[i], sp->slot_fn, sizeof(int) * sp->nslots, cudaMemcpyDeviceToDevice, st),
           "copy");
    SS_TRY(cudaMemcpyAsync(S->listed + t0, sp->listed, sizeof(int) * nt, cudaMemcpyDeviceToDevice, st), "copy");
    SS_TRY(cudaMemcpyAsync(S->exps + eoff[i], a->exps, sizeof(double) * sp->n_exps, cudaMemcpyDeviceToDevice, st),
           "copy");
    SS_TRY(cudaMemcpyAsync(S->norms + eoff[i], a->norms, sizeof(double) * sp->n_exps, cudaMemcpyDeviceToDevice, st),
           "copy");
    if (sp->n_contr)
      SS_TRY(cudaMemcpyAsync(S->contr + coff[i], a->contr, sizeof(double) * sp->n_contr, cudaMemcpyDeviceToDevice,
                             st), "copy");
    if (sp->n_rng)
      SS_TRY(cudaMemcpyAsync(S->rng + roff[i], a->rng, sizeof(int2) * sp->n_rng, cudaMemcpyDeviceToDevice, st),
             "copy");
    for (int l = 0; l <= kMaxL; ++l) {
      const int64_t ni = ioff[l][i + 1] - ioff[l][i];
      if (!ni) continue;
      BasisItem* dst = S->items[l] + ioff[l][i];
      SS_TRY(cudaMemcpyAsync(dst, sp->items[l], sizeof(BasisItem) * ni, cudaMemcpyDeviceToDevice, st), "copy");
      k_set_adjust_items<<<(unsigned)((ni + 255) / 256), 256, 0, st>>>(dst, ni, t0, soff[i], (int)eoff[i],
                                                                      (int)coff[i], (int)roff[i]);
    }
    for (int64_t t = 0; t <= nt; ++t) h_tso[(size_t)(t0 + t)] = sp->h_tso[(size_t)t] + soff[i];
    for (int64_t t = 0; t < nt; ++t) h_tile_mol[(size_t)(t0 + t)] = (int)i;
    const unsigned long long* P8;
    const int* eP;
    screen_mixed_p8(sp->mixed, 0, &P8, &eP);
    h_mols[i] = {P8, eP, sp->nbas, sp->V, sp->nbas};
    h_outs[i] = {a->acc, sp->V, sp->nbas, sp->gga ? 1 : 0, S->mem[i].d_ham, S->mem[i].d_exc_nel};
  }
  SS_TRY(cudaGetLastError(), "item offsets");
  SS_TRY(cudaMemcpyAsync(S->tso, h_tso.data(), sizeof(int64_t) * h_tso.size(), cudaMemcpyHostToDevice, st), "copy");
  SS_TRY(cudaMemcpyAsync(S->tile_mol, h_tile_mol.data(), sizeof(int) * h_tile_mol.size(), cudaMemcpyHostToDevice, st),
         "copy");
  SS_TRY(alloc(&S->mols, nm), "cudaMalloc");
  SS_TRY(alloc(&S->outs, nm), "cudaMalloc");
  SS_TRY(cudaMemcpyAsync(S->mols, h_mols.data(), sizeof(SetMolDev) * nm, cudaMemcpyHostToDevice, st), "copy");
  SS_TRY(cudaMemcpyAsync(S->outs, h_outs.data(), sizeof(SetOutDev) * nm, cudaMemcpyHostToDevice, st), "copy");
  // --- chunks: runs of whole tiles of one functional group --------------------
  size_t freeb = 0, totb = 0;
  SS_TRY(cudaMemGetInfo(&freeb, &totb), "cudaMemGetInfo");
  const bool any_gga = std::any_of(S->groups.begin(), S->groups.end(), [](const ScreenSet::Group& g) { return g.gga; });
  const int64_t per_slot = 128 * (8 + (any_gga ? 12 : 0)) + screen_mixed_bytes_per_slot();
  const int64_t per_tile = 128 * 8 * 8 + screen_mixed_bytes_per_tile() + 128 * 8 + 16;
  int64_t budget_slots = std::max<int64_t>((int64_t)(0.40 * (double)freeb) / per_slot, S->max_n);
  int64_t budget_tiles = std::max<int64_t>(1, (int64_t)(0.05 * (double)freeb) / per_tile);
  if (max_chunk_points > 0) budget_tiles = std::min(budget_tiles, std::max<int64_t>(1, max_chunk_points / 128));
  budget_tiles = std::min<int64_t>(budget_tiles, 1 << 16);
  std::vector<int64_t> boff((size_t)T + 1, 0);
  for (int64_t t = 0; t < T; ++t)
    boff[(size_t)t + 1] = boff[(size_t)t] + screen_mixed_bstages(h_tso[(size_t)t + 1] - h_tso[(size_t)t]);
  const int64_t budget_b = std::max<int64_t>((int64_t)(0.20 * (double)freeb) / screen_mixed_bytes_per_bstage(),
                                             screen_mixed_bstages(S->max_n));
  std::vector<SetSeg> h_segs;
  int64_t chunk_b = 0;
  {
    int64_t t0 = 0;
    auto close_chunk = [&](int64_t t1) {
      ScreenSet::Chunk c{};
      c.t0 = t0;
      c.t1 = t1;
      c.s0 = h_tso[(size_t)t0];
      c.group = mgroup[(size_t)h_tile_mol[(size_t)t0]];
      // item ranges: items are ordered by tile within and across contexts
      for (int l = 0; l <= kMaxL; ++l) {
        auto first_item = [&](int64_t t) {
          if (t >= T) return ioff[l][nm];
          const int m = h_tile_mol[(size_t)t];
          // the context's items before its tile t - toff[m]
          return ioff[l][(size_t)m] + S->mem[(size_t)m].sp->tile_item[l][(size_t)(t - toff[(size_t)m])];
        };
        c.i0[l] = first_item(t0);
        c.i1[l] = first_item(t1);
      }
      c.seg0 = (int64_t)h_segs.size();
      for (int64_t t = t0; t < t1;) {
        const int m = h_tile_mol[(size_t)t];
        const int64_t te = std::min(t1, toff[(size_t)m + 1]);
        h_segs.push_back({t - t0, te - t, m, 0});
        t = te;
      }
      c.nseg = (int64_t)h_segs.size() - c.seg0;
      S->chunks.push_back(c);
      S->chunk_tiles = std::max(S->chunk_tiles, t1 - t0);
      S->chunk_slots = std::max(S->chunk_slots, h_tso[(size_t)t1] - h_tso[(size_t)t0]);
      chunk_b = std::max(chunk_b, boff[(size_t)t1] - boff[(size_t)t0]);
      t0 = t1;
    };
    for (int64_t t = 0; t < T; ++t) {
      if (t == t0) continue;
      const bool new_group = mgroup[(size_t)h_tile_mol[(size_t)t]] != mgroup[(size_t)h_tile_mol[(size_t)t0]];
      const bool full = h_tso[(size_t)t + 1] - h_tso[(size_t)t0] > budget_slots || t + 1 - t0 > budget_tiles ||
                        boff[(size_t)t + 1] - boff[(size_t)t0] > budget_b;
      if (new_group || full) close_chunk(t);
    }
    close_chunk(T);
  }
  SS_TRY(alloc(&S->segs, h_segs.size()), "cudaMalloc");
  SS_TRY(cudaMemcpyAsync(S->segs, h_segs.data(), sizeof(SetSeg) * h_segs.size(), cudaMemcpyHostToDevice, st), "copy");
  SS_TRY(alloc(&S->b_off, boff.size()), "cudaMalloc");
  SS_TRY(cudaMemcpyAsync(S->b_off, boff.data(), sizeof(int64_t) * boff.size(), cudaMemcpyHostToDevice, st), "copy");
  // --- chunk buffers -----------------------------------------------------------
  const size_t rows = (size_t)(S->chunk_slots + kSlack) * 128;
  SS_TRY(alloc(&S->phi, rows), "cudaMalloc (phi)");
  SS_TRY(cudaMemsetAsync(S->phi, 0, sizeof(double) * rows, st), "memset");
  if (any_gga) {
    SS_TRY(alloc(&S->gx, rows), "cudaMalloc (grad phi)");
    SS_TRY(alloc(&S->gy, rows), "cudaMalloc (grad phi)");
    SS_TRY(alloc(&S->gz, rows), "cudaMalloc (grad phi)");
    SS_TRY(cudaMemsetAsync(S->gx, 0, sizeof(float) * rows, st), "memset");
    SS_TRY(cudaMemsetAsync(S->gy, 0, sizeof(float) * rows, st), "memset");
    SS_TRY(cudaMemsetAsync(S->gz, 0, sizeof(float) * rows, st), "memset");
  }
  SS_TRY(alloc(&S->pt, 8 * (size_t)S->chunk_tiles * 128), "cudaMalloc");
  SS_TRY(alloc(&S->partial, 2 * (size_t)S->chunk_tiles), "cudaMalloc");
  SS_TRY(alloc(&S->pmax, (size_t)S->chunk_tiles * 128), "cudaMalloc");
  SS_TRY(cudaStreamSynchronize(st), "set-up");
  ScreenMixedInput mi;
  mi.nbas = 1;  // the members' own density-matrix digits are used
  mi.ldc = 1;
  mi.gga = any_gga;
  mi.nspin = 1;
  mi.chunk_slots = S->chunk_slots + kSlack;
  mi.chunk_tiles = S->chunk_tiles;
  mi.max_n = S->max_n;
  mi.chunk_bstages = chunk_b;
  mi.b_off = S->b_off;
  std::string e2;
  if (int st2 = screen_mixed_create(&S->mixed, mi, e2)) return fail(st2, e2);
#undef SS_TRY
  *out = S;
  return PGXC_OK;
}

int screen_set_run(ScreenSet* S, cudaStream_t st, std::string& err) {
  const int64_t cp = S->chunk_tiles * 128;
  int64_t launches = 0;
  for (const ScreenSet::Chunk& c : S->chunks) {
    const ScreenSet::Group& g = S->groups[(size_t)c.group];
    const bool gga = g.gga;
    const int64_t t0 = c.t0, nt = c.t1 - c.t0, s0 = c.s0;
    float* gxc = gga ? S->gx : nullptr;
    float* gyc = gga ? S->gy : nullptr;
    float* gzc = gga ? S->gz : nullptr;
    cudaMemsetAsync(S->pmax, 0, sizeof(unsigned long long) * nt * 128, st);
    auto launch_l = [&](auto Lc) {
      constexpr int L = decltype(Lc)::value;
      const int64_t i0 = c.i0[L], n = c.i1[L] - c.i0[L];
      if (n <= 0) return;
      const unsigned nb = (unsigned)std::min<int64_t>(n, (int64_t)S->nsm * kBasisBlocksPerSM);
      if (gga)
        k_basis_items<L, true, float><<<nb, 128, 0, st>>>(S->items[L] + i0, n, S->exps, S->norms, S->contr, S->rng,
                                                          S->sa, S->qx, S->qy, S->qz, s0, t0, S->phi, gxc, gyc, gzc,
                                                          S->pmax);
      else
        k_basis_items<L, false, float><<<nb, 128, 0, st>>>(S->items[L] + i0, n, S->exps, S->norms, S->contr, S->rng,
                                                           S->sa, S->qx, S->qy, S->qz, s0, t0, S->phi, (float*)nullptr,
                                                           (float*)nullptr, (float*)nullptr, S->pmax);
      ++launches;
    };
    launch_l(std::integral_constant<int, 0>());
    launch_l(std::integral_constant<int, 1>());
    launch_l(std::integral_constant<int, 2>());
    launch_l(std::integral_constant<int, 3>());
    if (gga) k_pad_zero<true, float><<<(unsigned)nt, 128, 0, st>>>(S->tso, S->listed, t0, s0, S->phi, gxc, gyc, gzc);
    else k_pad_zero<false, float><<<(unsigned)nt, 128, 0, st>>>(S->tso, S->listed, t0, s0, S->phi, (float*)nullptr,
                                                                (float*)nullptr, (float*)nullptr);
    ++launches;
    screen_mixed_set_gga(S->mixed, gga);
    launches += screen_mixed_basis(S->mixed, S->tso, S->slot_fn, t0, nt, s0, S->phi, S->pmax, 0, 0, st, S->tile_mol,
                                   S->mols);
    double* q = S->pt;
    BuildArgs b{};
    b.xc = g.xc;
    b.w = S->qw;
    b.rho = q;
    b.grx = q + cp;
    b.gry = q + 2 * cp;
    b.grz = q + 3 * cp;
    b.A = q + 4 * cp;
    b.Bx = q + 5 * cp;
    b.By = q + 6 * cp;
    b.Bz = q + 7 * cp;
    b.partial = S->partial;
    launches += screen_mixed_density(S->mixed, S->tso, S->slot_fn, t0, nt, s0, S->phi, gxc, gyc, gzc, b.rho, b.grx,
                                     b.gry, b.grz, 0, 0, st);
    launch_functional_tiles(b, t0 * 128, nt, gga, st);
    k_set_sum<<<(unsigned)c.nseg, 128, 0, st>>>(S->partial, S->segs + c.seg0, S->outs);
    launches += 2;
    launches += screen_mixed_potential(S->mixed, S->tso, S->slot_fn, nullptr, t0, nt, s0, 0, S->phi, gxc, gyc, gzc, b.A,
                                       b.Bx, b.By, b.Bz, nullptr, 0, st, nullptr, nullptr, S->tile_mol, S->mols);
  }
  k_set_pack<<<(unsigned)S->mem.size(), 256, 0, st>>>(S->outs);
  ++launches;
  S->launches = launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("set build: ") + cudaGetErrorString(e);
    return PGXC_ECUDA;
  }
  return PGXC_OK;
}

int screen_set_error_flag(ScreenSet* S, cudaStream_t st, int* flag) { return screen_mixed_error_flag(S->mixed, st, flag); }

int screen_set_prepare_member(ScreenPlan* sp, const double* P, int64_t ldc, cudaStream_t st) {
  if (cudaMemsetAsync(sp->V, 0, sizeof(double) * sp->nbas * sp->nbas, st) != cudaSuccess) return PGXC_ECUDA;
  screen_mixed_prepare(sp->mixed, P, ldc, 0, st);
  return cudaGetLastError() == cudaSuccess ? PGXC_OK : PGXC_ECUDA;
}

bool screen_set_eligible(const ScreenPlan* sp) { return sp->mixed && sp->ispin == 1 && !sp->keep && !sp->mgga; }

}  // namespace pgxc
