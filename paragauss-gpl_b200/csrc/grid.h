// grid.h -- device-built atom-centred grids and the device Morton order.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace pgxc {

// The Lebedev-McLaren rule with npts points (INIGRD, modules/grid_module.f90
// :1359-2100) as x, y, z, w quadruples; 0, or -1 when no rule has npts points.
int lebedev_rule(int npts, std::vector<double>& xyzw);

// Radial shells RADIALGRID keeps of a Pople grid with nradpts points and
// scale rcur: those with r < 40 bohr (modules/grid_module.f90:1279-1285).
int64_t radial_shells(int nradpts, double rcur);

// The product grid of natm atoms: points off[a] .. off[a+1]-1 belong to atom
// a (shell-major, nang angular points per shell); SoA outputs of n points.
cudaError_t launch_atomic_grid(int natm, const double* d_atoms, const int64_t* d_off, const double* d_rcur,
                               const int* d_nrad, const double* d_ang, int nang, int64_t n, double* gx, double* gy,
                               double* gz, double* gw, int* owner, cudaStream_t st);

// perm[0 .. n-1] = the points in Morton order of their coordinates (ties by
// index), perm[n .. total-1] = -1; synchronises st.
cudaError_t morton_perm_device(const double* px, const double* py, const double* pz, int64_t n, int64_t total,
                               int64_t* perm, cudaStream_t st);

}  // namespace pgxc
