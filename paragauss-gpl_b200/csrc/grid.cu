// grid.cu -- atom-centred integration grids built on the device, and the
// Morton order of a grid's points (used to cut the screened build's tiles).
//
// The grid is the reference's grid_main_calc without pruning
// (modules/grid_module.f90:357-504): per atom, the Pople radial grid of
// RADIALGRID (:1246-1301) times a Lebedev-McLaren angular rule of INIGRD
// (:1359-2100), points ordered atom -> radial shell -> angular point, one-centre
// weights w_ang * w_rad * 4 pi (:425-432).  The angular rule is not rotated
// (the orientation the reference uses when weight gradients are on).
//
// The arithmetic is written with explicit round-to-nearest operations in the
// order the reference writes it, (I/RHNI)**2, 2*RCUR**3*RHN*(I/RHNI)**5/RHNI**2
// with the integer powers as products, so the device grid equals, bit for
// bit, the host restatement in pgxc/grid.py that the tests use.
#include <algorithm>
#include <array>
#include <cmath>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "grid.h"

namespace pgxc {

namespace {

// ---------------------------------------------------------------------------
// Lebedev-McLaren rules: the published orbit parameters and weights exactly
// as INIGRD holds them (a table of published constants has to be alike).
// ---------------------------------------------------------------------------
enum OrbitKind { kA1, kA2, kA3, kB, kC, kD };
struct OrbitSpec {
  OrbitKind kind;
  double p1, p2, w;
};
struct RuleSpec {
  int npts;
  std::vector<OrbitSpec> orbits;
};

const std::vector<RuleSpec>& rules() {
  static const std::vector<RuleSpec> r = {
      {6, {{kA1, 0, 0, 1.0 / 6.0}}},
      {8, {{kA3, 0, 0, 1.0 / 8.0}}},
      {12, {{kA2, 0, 0, 1.0 / 12.0}}},
      {14, {{kA1, 0, 0, 8.0 / 120.0}, {kA3, 0, 0, 9.0 / 120.0}}},
      {26, {{kA1, 0, 0, 40.0 / 840.0}, {kA2, 0, 0, 32.0 / 840.0}, {kA3, 0, 0, 27.0 / 840.0}}},
      {38, {{kA1, 0, 0, 1.0 / 105.0}, {kA3, 0, 0, 9.0 / 280.0}, {kC, 1.0 / 6.0, 0, 1.0 / 35.0}}},
      {50,
       {{kA1, 0, 0, 4.0 / 315.0},
        {kA2, 0, 0, 64.0 / 2835.0},
        {kA3, 0, 0, 27.0 / 1280.0},
        {kB, 3.0 / std::sqrt(11.0), 0, 14641.0 / 725760.0}}},
      {78,
       {{kA1, 0, 0, 0.0138665921047},
        {kB, 0.914152532416, 0, 0.0130509318626},
        {kB, 0.359236381200, 0, 0.0132064232231},
        {kC, 0.206339716383, 0, 0.0119426635549}}},
      {86,
       {{kA1, 0, 0, 8.0 / 693.0},
        {kA3, 0, 0, 0.0119439090859},
        {kB, 0.852518311701, 0, 0.0111105557106},
        {kB, 0.189063552885, 0, 0.0118765012945},
        {kC, 0.120441650315, 0, 0.0118123037469}}},
      {110,
       {{kA1, 0, 0, 0.00382827049494},
        {kA3, 0, 0, 0.00979373751249},
        {kB, 0.965124035087, 0, 0.00821173728319},
        {kB, 0.828769981253, 0, 0.00959547133607},
        {kB, 0.215957291846, 0, 0.00994281489118},
        {kC, 3.0 / 17.0, 0, 19652.0 / 2027025.0}}},
      {146,
       {{kA1, 0, 0, 1856.0 / 3095235.0},
        {kA2, 0, 0, 606208.0 / 82219995.0},
        {kA3, 0, 0, 6490935.0 / 900204032.0},
        {kB, 0.974888643677, 0, 7.57439415905e-03},
        {kB, 0.807089818360, 0, 6.75382948631e-03},
        {kB, 0.291298882210, 0, 7.11635549312e-03},
        {kD, 0.140355381171, 0.449332832327, 1773593.0 / 253693440.0}}},
      {194,
       {{kA1, 0, 0, 1.78234044724e-03},
        {kA2, 0, 0, 5.71690594998e-03},
        {kA3, 0, 0, 5.57338317884e-03},
        {kB, 0.777493219315, 0, 5.51877146727e-03},
        {kB, 0.912509096867, 0, 5.15823771181e-03},
        {kB, 0.314196994183, 0, 5.60870408259e-03},
        {kB, 0.982972302707, 0, 4.10677702817e-03},
        {kC, 2.0 / 19.0, 0, 5.05184606462e-03},
        {kD, 0.159041710538, 0.525118572443, 5.53024891623e-03}}},
      {302,
       {{kA1, 0, 0, 8.54591172878e-04},
        {kA3, 0, 0, 3.59911928502e-03},
        {kB, 0.129238672710, 0, 3.65004580768e-03},
        {kB, 0.371034178385, 0, 3.60482260142e-03},
        {kB, 0.743452042987, 0, 3.57672966173e-03},
        {kB, 0.867643624544, 0, 3.44978842429e-03},
        {kB, 0.949454317226, 0, 3.10895312238e-03},
        {kB, 0.990705621379, 0, 2.35210141366e-03},
        {kC, 0.220093335298, 0, 3.60082093222e-03},
        {kC, 0.650272754659e-01, 0, 2.98234496317e-03},
        {kD, 0.800072749407, 0.544867737258, 3.57154055427e-03},
        {kD, 0.902442529533, 0.412772408317, 3.39231220501e-03}}},
  };
  return r;
}

using P3 = std::array<double, 3>;

// the 8 sign triples in INIGRD's loop order (I outer, K inner)
const double kSign[8][3] = {{-1, -1, -1}, {-1, -1, 1}, {-1, 1, -1}, {-1, 1, 1},
                            {1, -1, -1},  {1, -1, 1},  {1, 1, -1},  {1, 1, 1}};

// 12 points with a, b on two axes (xy, xz, yz; signs ++, +-, -+, --)
void two_axis(double a, double b, std::vector<P3>& out) {
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  const double sg[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
  for (auto& pr : pairs)
    for (auto& s : sg) {
      P3 v = {0.0, 0.0, 0.0};
      v[pr[0]] = s[0] * a;
      v[pr[1]] = s[1] * b;
      out.push_back(v);
    }
}

// the sign triples applied to t1, then t2, then t3
void three_types(const P3& t1, const P3& t2, const P3& t3, std::vector<P3>& out) {
  for (const P3* t : {&t1, &t2, &t3})
    for (auto& s : kSign) out.push_back({s[0] * (*t)[0], s[1] * (*t)[1], s[2] * (*t)[2]});
}

void orbit(const OrbitSpec& o, std::vector<P3>& out) {
  switch (o.kind) {
    case kA1:
      out.insert(out.end(), {{0, 0, 1}, {0, 0, -1}, {0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}});
      break;
    case kA2: {
      const double r = 1.0 / std::sqrt(2.0);
      two_axis(r, r, out);
      break;
    }
    case kA3: {
      const double r = 1.0 / std::sqrt(3.0);
      for (auto& s : kSign) out.push_back({s[0] * r, s[1] * r, s[2] * r});
      break;
    }
    case kB: {
      const double m = o.p1, l = std::sqrt((1.0 - m * m) / 2.0);
      three_types({l, l, m}, {l, m, l}, {m, l, l}, out);
      break;
    }
    case kC: {
      const double d = std::sqrt(1.0 - 4.0 * o.p1);
      const double p = std::sqrt((1.0 + d) / 2.0), q = std::sqrt((1.0 - d) / 2.0);
      two_axis(p, q, out);
      two_axis(q, p, out);
      break;
    }
    case kD: {
      const double u = o.p1, w = o.p2, r = std::sqrt(1.0 - u * u - w * w);
      std::vector<P3> first;
      three_types({u, w, r}, {w, r, u}, {r, u, w}, first);
      out.insert(out.end(), first.begin(), first.end());
      for (const P3& v : first) out.push_back({v[0], v[2], v[1]});
      break;
    }
  }
}

// ---------------------------------------------------------------------------
// device kernels
// ---------------------------------------------------------------------------
// Point q: atom a (off[a] <= q < off[a+1]), radial shell I = (q - off[a]) / nang + 1
// (1-based, as RADIALGRID counts), angular point j.
__global__ void k_atomic_grid(int natm, const double* __restrict__ atoms, const int64_t* __restrict__ off,
                              const double* __restrict__ rcur, const int* __restrict__ nradpts,
                              const double* __restrict__ ang, int nang, double fourpi, int64_t n,
                              double* __restrict__ gx, double* __restrict__ gy, double* __restrict__ gz,
                              double* __restrict__ gw, int* __restrict__ owner) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = natm;  // largest a with off[a] <= q
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= q) lo = mid;
      else hi = mid;
    }
    const int a = lo;
    const int64_t loc = q - off[a];
    const int I = (int)(loc / nang) + 1, j = (int)(loc % nang);
    const double R = rcur[a];
    const double rhn = (double)(nradpts[a] + 1);
    const double rhni = __dsub_rn(rhn, (double)I);
    const double t = __ddiv_rn((double)I, rhni);
    const double t2 = __dmul_rn(t, t);
    const double r = __dmul_rn(R, t2);
    const double r3 = __dmul_rn(__dmul_rn(R, R), R);
    const double t5 = __dmul_rn(__dmul_rn(t2, t2), t);
    const double wr =
        __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, r3), rhn), t5), __dmul_rn(rhni, rhni));
    gx[q] = __dadd_rn(__dmul_rn(r, ang[4 * j]), atoms[3 * a]);
    gy[q] = __dadd_rn(__dmul_rn(r, ang[4 * j + 1]), atoms[3 * a + 1]);
    gz[q] = __dadd_rn(__dmul_rn(r, ang[4 * j + 2]), atoms[3 * a + 2]);
    gw[q] = __dmul_rn(__dmul_rn(wr, ang[4 * j + 3]), fourpi);
    owner[q] = a;
  }
}

// --- Morton order -----------------------------------------------------------
__global__ void k_bounds(const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
                         int64_t n, double* __restrict__ part) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v[3] = {px[i], py[i], pz[i]};
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], v[d]);
      hi[d] = fmax(hi[d], v[d]);
    }
  }
  __shared__ double s[6][256];
  for (int d = 0; d < 3; ++d) {
    s[d][threadIdx.x] = lo[d];
    s[3 + d][threadIdx.x] = hi[d];
  }
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + o]);
        s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) part[blockIdx.x * 6 + threadIdx.x] = s[threadIdx.x][0];
}

__device__ __forceinline__ unsigned long long spread3(unsigned long long v) {  // 21 bits -> every third bit
  v &= 0x1fffffull;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}

// key of point i: bit-interleaved 21-bit cell coordinates (x lowest)
__global__ void k_morton_keys(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, int64_t n, const double* __restrict__ part, int nparts,
                              unsigned long long* __restrict__ key, int64_t* __restrict__ idx) {
  double lo[3], span[3];
  for (int d = 0; d < 3; ++d) {
    double l = INFINITY, h = -INFINITY;
    for (int b = 0; b < nparts; ++b) {
      l = fmin(l, part[b * 6 + d]);
      h = fmax(h, part[b * 6 + 3 + d]);
    }
    lo[d] = l;
    span[d] = __dsub_rn(h, l);
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v[3] = {px[i], py[i], pz[i]};
    unsigned long long k = 0;
    for (int d = 0; d < 3; ++d) {
      const double u = span[d] > 0 ? __ddiv_rn(__dsub_rn(v[d], lo[d]), span[d]) : 0.0;
      const double c = fmin(2097151.0, fmax(0.0, __dmul_rn(u, 2097151.0)));
      k |= spread3((unsigned long long)c) << d;
    }
    key[i] = k;
    idx[i] = i;
  }
}

__global__ void k_pad_perm(int64_t* __restrict__ perm, int64_t n, int64_t total) {
  const int64_t i = n + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) perm[i] = -1;
}

}  // namespace

int lebedev_rule(int npts, std::vector<double>& xyzw) {
  for (const RuleSpec& r : rules()) {
    if (r.npts != npts) continue;
    xyzw.clear();
    for (const OrbitSpec& o : r.orbits) {
      std::vector<P3> pts;
      orbit(o, pts);
      for (const P3& v : pts) xyzw.insert(xyzw.end(), {v[0], v[1], v[2], o.w});
    }
    return (int)(xyzw.size() / 4) == npts ? 0 : -1;
  }
  return -1;
}

int64_t radial_shells(int nradpts, double rcur) {
  // RADIALGRID: the largest I <= NRADPTS with r(I) < RAD_LIMIT = 40
  const double rhn = (double)nradpts + 1.0;
  int I = nradpts;
  for (; I >= 1; --I) {
    const double rhni = rhn - (double)I;
    const double t = (double)I / rhni;
    if (rcur * (t * t) < 40.0) break;
  }
  return std::max(I, 0);
}

cudaError_t launch_atomic_grid(int natm, const double* d_atoms, const int64_t* d_off, const double* d_rcur,
                               const int* d_nrad, const double* d_ang, int nang, int64_t n, double* gx, double* gy,
                               double* gz, double* gw, int* owner, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned nb = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32);
  k_atomic_grid<<<nb, 256, 0, st>>>(natm, d_atoms, d_off, d_rcur, d_nrad, d_ang, nang, 16.0 * std::atan(1.0), n, gx,
                                    gy, gz, gw, owner);
  return cudaGetLastError();
}

cudaError_t morton_perm_device(const double* px, const double* py, const double* pz, int64_t n, int64_t total,
                               int64_t* perm, cudaStream_t st) {
  constexpr int kParts = 148;
  double* part = nullptr;
  unsigned long long *key = nullptr, *key2 = nullptr;
  int64_t* idx = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaError_t e = cudaMalloc(&part, sizeof(double) * 6 * kParts);
  if (e == cudaSuccess) e = cudaMalloc(&key, sizeof(unsigned long long) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(&key2, sizeof(unsigned long long) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(&idx, sizeof(int64_t) * std::max<int64_t>(n, 1));
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, idx, perm, n, 0, 64, st);
  if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 1));
  if (e == cudaSuccess) {
    k_bounds<<<kParts, 256, 0, st>>>(px, py, pz, n, part);
    const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32));
    k_morton_keys<<<nb, 256, 0, st>>>(px, py, pz, n, part, kParts, key, idx);
    e = cudaGetLastError();
  }
  // stable radix sort: equal keys keep ascending point index (the host order's tie-break)
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, idx, perm, n, 0, 64, st);
  if (e == cudaSuccess && total > n)
    k_pad_perm<<<(unsigned)((total - n + 255) / 256), 256, 0, st>>>(perm, n, total);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(part);
  cudaFree(key);
  cudaFree(key2);
  cudaFree(idx);
  cudaFree(tmp);
  return e;
}

}  // namespace pgxc
