// Whole steps of a small microenvironment in one cooperative launch.
//
// A field of up to ~1M voxel-densities with at most 64 points per axis costs
// more in kernel start-up than in work when every phase of a step is its own
// launch (7 launches per step at 50^3 x 1).  Here every step runs inside one
// launch over all SMs, as phases separated by grid-wide barriers of a
// cooperative launch (all blocks are resident, so each barrier completes):
//   sources: per bulk entry its update (BioFVM_microenvironment.cpp:603-609)
//            and then its voxel's agents in list order
//            (BioFVM_basic_agent.cpp:234-235); per agent voxel without a bulk
//            entry its agents;
//   x, y, z: each thread solves whole (line, density) items in its own
//            column of shared memory (points blockDim.x elements apart, so
//            the threads of a warp hit different banks); as a line is loaded, its Dirichlet nodes take their
//            values (BioFVM_microenvironment.cpp:192-197, before each axis:
//            BioFVM_solvers.cpp:177, 207, 241): a 64-bit mask per line marks
//            the nodes, whose values sit in a field-shaped array.
// Offsets are 32-bit: the path is for fields of at most 2^20 elements.
// Every voxel lies on exactly one line per axis, so this equals the
// reference's whole-field passes.  Lines are solved with the reference's
// recurrence (BioFVM_solvers.cpp:186-200) using precomputed reciprocals of
// the denominators (a multiply instead of a divide), within 1e-15 of the
// divided form.
#pragma once

#include <cooperative_groups.h>

#include "bfvm_kernels.cuh"

namespace bfvm {

struct GridStepArgs {
  double* p;  // [nz][ny][nx][S]
  int nx, ny, nz, S;
  int nsteps;
  double dt;
  bool bulk, cells;
  // per axis: 1/denominator [n][S], cx [n][S], c1 [S]
  const double* rd[3];
  const double* cx[3];
  const double* c1[3];
  // per voxel: its bulk entry and its first agent in the sorted list, or -1
  const int* bulk_map;
  const int* ag_map;
  // Dirichlet nodes: per axis and line a mask of the points that are nodes
  // (lines numbered x: k*ny + j, y: k*nx + i, z: j*nx + i), and the node
  // values at their places in a field-shaped array [N][S]
  bool dirichlet;
  const unsigned long long* dir_mask[3];
  const double* dir_field;
  int64_t nbulk;
  const int64_t* bulk_vox;  // [E] ascending
  const double* bulk_st;    // [E][S] S*T
  const double* bulk_su;    // [E][S] U+S
  int64_t nagents;
  const uint64_t* ag_key;  // sorted voxel keys (stable in list order)
  const int* ag_idx;       // list position of each sorted entry
  const double* ag_t1;     // [A][S] in list order
  const double* ag_t2;
};

// The agents of one voxel, from its first sorted entry r, in list order.
__device__ __forceinline__ double grid_cells(const GridStepArgs& a, double x, int r, uint64_t vox,
                                             int s) {
  do {
    const int64_t ai = __ldg(a.ag_idx + r);
    x = cell_update(x, __ldg(a.ag_t1 + ai * a.S + s), __ldg(a.ag_t2 + ai * a.S + s));
    ++r;
  } while (r < a.nagents && __ldg(a.ag_key + r) == vox);
  return x;
}

// Bulk then cell updates of every voxel that has either.
__device__ __forceinline__ void grid_sources(const GridStepArgs& a, int64_t first,
                                             int64_t stride) {
  const int S = a.S;
  const int64_t nb = a.bulk ? a.nbulk * S : 0;
  const int64_t na = a.cells ? a.nagents * S : 0;
  for (int64_t w = first; w < nb + na; w += stride) {
    if (w < nb) {
      const int64_t e = w / S;
      const int s = (int)(w - e * S);
      const int64_t vox = __ldg(a.bulk_vox + e);
      double* q = a.p + vox * S + s;
      double x = bulk_update(*q, __ldg(a.bulk_st + w), __ldg(a.bulk_su + w), a.dt);
      if (a.cells) {
        const int r = __ldg(a.ag_map + vox);
        if (r >= 0) x = grid_cells(a, x, r, (uint64_t)vox, s);
      }
      *q = x;
    } else {
      const int64_t r = (w - nb) / S;
      const int s = (int)(w - nb - r * S);
      const uint64_t vox = __ldg(a.ag_key + r);
      if (r > 0 && __ldg(a.ag_key + r - 1) == vox) continue;  // not the voxel's first agent
      if (a.bulk && __ldg(a.bulk_map + vox) >= 0) continue;   // done with its bulk entry
      double* q = a.p + (int64_t)vox * S + s;
      *q = grid_cells(a, *q, (int)r, vox, s);
    }
  }
}

// The lines of one axis: each thread takes (line, density) items.
template <int AX>
__device__ __forceinline__ void grid_axis(const GridStepArgs& a, double* col, int first,
                                          int stride) {
  const int S = a.S;
  const int T = blockDim.x;  // shared-memory elements between a column's points
  const int plane = a.nx * a.ny;
  const int n = AX == 0 ? a.nx : (AX == 1 ? a.ny : a.nz);
  const int st = (AX == 0 ? 1 : (AX == 1 ? a.nx : plane)) * S;  // field elements between points
  const int items = plane * a.nz / n * S;
  const double* __restrict__ rd = a.rd[AX];
  const double* __restrict__ cx = a.cx[AX];
  for (int l = first; l < items; l += stride) {
    const int s = l % S;
    const int line = l / S;
    int base;  // voxel of point 0
    if (AX == 0)
      base = line * a.nx;
    else if (AX == 1)
      base = (line / a.nx) * plane + line % a.nx;
    else
      base = line;
    double* q = a.p + base * S + s;
    const double* dq = a.dir_field + base * S + s;
    const unsigned long long nodes = a.dirichlet ? __ldg(a.dir_mask[AX] + line) : 0ull;
    // branch-free loads (both values, then a select) so that they overlap
    if (nodes == 0ull) {
#pragma unroll 8
      for (int k = 0; k < n; ++k) col[k * T] = q[k * st];
    } else {
#pragma unroll 8
      for (int k = 0; k < n; ++k) {
        const double x = q[k * st], d = __ldg(dq + k * st);
        col[k * T] = ((nodes >> k) & 1ull) ? d : x;
      }
    }
    // forward: p_0 /= d_0; p_k = (p_k + c1 p_{k-1}) / d_k (as multiplies)
    const double c1 = __ldg(a.c1[AX] + s);
    double prev = col[0] * __ldg(rd + s);
    col[0] = prev;
#pragma unroll 8
    for (int k = 1; k < n; ++k) {
      prev = (col[k * T] + c1 * prev) * __ldg(rd + k * S + s);
      col[k * T] = prev;
    }
    // back: p_k -= cx_k p_{k+1}, straight to the field
    q[(n - 1) * st] = prev;
#pragma unroll 8
    for (int k = n - 2; k >= 0; --k) {
      prev = col[k * T] - __ldg(cx + k * S + s) * prev;
      q[k * st] = prev;
    }
  }
}

// nsteps whole steps; launched cooperatively (every block resident) with
// blockDim.x * (most points per axis) doubles of dynamic shared memory.
__global__ void __launch_bounds__(128) grid_steps_kernel(const GridStepArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double grid_cols[];
  double* col = grid_cols + threadIdx.x;
  const int first = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int step = 0; step < a.nsteps; ++step) {
    if (a.bulk || a.cells) {
      grid_sources(a, first, stride);
      grid.sync();
    }
    grid_axis<0>(a, col, first, stride);
    grid.sync();
    grid_axis<1>(a, col, first, stride);
    grid.sync();
    grid_axis<2>(a, col, first, stride);
    grid.sync();
  }
}

// Dense voxel maps of the bulk entries and of the first agent of each voxel
// in the sorted list (both -1 beforehand), and the Dirichlet nodes' line
// masks (0 beforehand) and values at their places in the field.
static __global__ void grid_maps_kernel(int* __restrict__ bulk_map, int* __restrict__ ag_map,
                                        int64_t nbulk, const int64_t* __restrict__ bulk_vox,
                                        int64_t nagents, const uint64_t* __restrict__ ag_key,
                                        int64_t ndir, const int64_t* __restrict__ dir_vox,
                                        const double* __restrict__ dir_val,
                                        unsigned long long* __restrict__ mx,
                                        unsigned long long* __restrict__ my,
                                        unsigned long long* __restrict__ mz,
                                        double* __restrict__ dir_field, int nx, int ny, int S) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
       i < nbulk || i < nagents || i < ndir; i += stride) {
    if (i < nbulk) bulk_map[bulk_vox[i]] = (int)i;
    if (i < nagents && (i == 0 || ag_key[i] != ag_key[i - 1])) ag_map[ag_key[i]] = (int)i;
    if (i < ndir) {
      const int64_t v = dir_vox[i];
      const int64_t plane = (int64_t)nx * ny;
      const int64_t k = v / plane, ij = v - k * plane, j = ij / nx, ii = ij - j * nx;
      atomicOr(mx + v / nx, 1ull << ii);
      atomicOr(my + k * nx + ii, 1ull << j);
      atomicOr(mz + ij, 1ull << k);
      for (int s = 0; s < S; ++s) dir_field[v * S + s] = dir_val[i * S + s];
    }
  }
}

}  // namespace bfvm
