// Whole steps of a small microenvironment in one cooperative launch.
//
// A field of up to ~1M voxel-densities with at most 64 points per axis costs
// more in kernel start-up than in work when every phase of a step is its own
// launch (7 launches per step at 50^3 x 1).  Here every step runs inside one
// launch over all SMs, as phases separated by grid-wide barriers of a
// cooperative launch (all blocks are resident, so each barrier completes;
// after the first step the sources ride on the z phase of the step before):
//   sources: per bulk entry its update (BioFVM_microenvironment.cpp:603-609)
//            and then its voxel's agents in list order
//            (BioFVM_basic_agent.cpp:234-235); per agent voxel without a bulk
//            entry its agents;
//   x, y, z: tiles of TW lines x NC chunks of 4 or 8 points per block (as the
//            register sweep kernel: chunk-local passes, the chunks' carries
//            folded through shared memory, fix-ups); as a chunk is loaded, its
//            Dirichlet nodes take their values (BioFVM_microenvironment.cpp:
//            192-197, before each axis: BioFVM_solvers.cpp:177, 207, 241): a
//            64-bit mask per line marks the nodes, whose values sit in a
//            field-shaped array.
// Every voxel lies on exactly one line per axis, so this equals the
// reference's whole-field passes.  Lines are solved with the sweep kernels'
// per-point tables (1/denominator, forward and backward slopes), within
// 1e-12 of the reference's divisions.
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
  // per axis: the sweep kernels' per-point tables [n][S] and c1 [S]
  AxisCoef<double> coef[3];
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

// The lines of one axis in tiles of TW columns x NC chunks (TW = blockDim.x /
// NC); columns are (line, density) pairs numbered as in lod_sweep_kernel.
// sm holds 4 * blockDim.x values for the chunks' forward and backward carries.
// With sources_after (z only), each stored point first takes the next step's
// bulk and cell updates: every voxel lies on exactly one z chunk, so the
// thread that solved it is the only one to touch it before the next x phase.
template <int AX, int CH>
__device__ __forceinline__ void grid_axis(const GridStepArgs& a, double* sm,
                                          bool sources_after = false) {
  const int S = a.S;
  const int64_t plane = (int64_t)a.nx * a.ny;
  const int n = AX == 0 ? a.nx : (AX == 1 ? a.ny : a.nz);
  const int64_t C = AX == 0 ? S : (AX == 1 ? (int64_t)a.nx * S : plane * S);
  const int64_t outer_stride = AX == 0 ? (int64_t)a.nx * S : (AX == 1 ? plane * S : 0);
  const int64_t ls = AX == 0 ? S : (AX == 1 ? (int64_t)a.nx * S : plane * S);
  const int64_t ncols = plane * a.nz / n * S;
  const int NC = (n + CH - 1) / CH;
  const int TW = blockDim.x / NC;
  const int tx = threadIdx.x % TW;
  const int c = threadIdx.x / TW;  // chunk; threads past NC chunks idle
  const bool in_tile = c < NC;
  const int k0 = c * CH;
  double* sQ = sm;  // [NC][TW] forward chunk end values
  double* sP = sQ + NC * TW;
  double* sX = sP + NC * TW;  // backward chunk start values
  double* sR = sX + NC * TW;
  const AxisCoef<double> cf = a.coef[AX];
  const int64_t ntiles = (ncols + TW - 1) / TW;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t vcol = tile * TW + tx;
    const bool active = in_tile && vcol < ncols;
    const int len = active ? max(0, min(CH, n - k0)) : 0;
    double* ptr = a.p;
    const double* dptr = a.dir_field;
    int s = 0;
    unsigned long long nodes = 0ull;
    if (active) {
      const int64_t outer = vcol / C;
      const int64_t col = vcol - outer * C;
      const int64_t off = outer * outer_stride + col + (int64_t)k0 * ls;
      ptr = a.p + off;
      dptr = a.dir_field + off;
      s = (int)(col % S);
      if (a.dirichlet) nodes = __ldg(a.dir_mask[AX] + vcol / S) >> k0;
    }
    double v[CH];
#pragma unroll
    for (int m = 0; m < CH; ++m)
      v[m] = (m < len) ? (((nodes >> m) & 1ull) ? __ldg(dptr + m * ls) : ptr[m * ls]) : 0.0;
    const double* c_inv = cf.inv_den + (int64_t)k0 * S + s;
    const double* c_fwd = cf.fwd + (int64_t)k0 * S + s;
    const double* c_bwd = cf.bwd + (int64_t)k0 * S + s;
    // forward elimination, chunk-local with carry-in 0
    const double c1 = active ? __ldg(cf.c1 + s) : 0.0;
    double q = 0.0, P = 1.0;
#pragma unroll
    for (int m = 0; m < CH; ++m) {
      if (m < len) {
        q = (v[m] + c1 * q) * __ldg(c_inv + m * S);
        P = P * __ldg(c_fwd + m * S);
        v[m] = q;
      }
    }
    if (in_tile) {
      sQ[c * TW + tx] = q;
      sP[c * TW + tx] = P;
    }
    __syncthreads();
    if (c > 0 && len > 0) {
      double carry = 0.0;
      for (int cc = 0; cc < c; ++cc) carry = sP[cc * TW + tx] * carry + sQ[cc * TW + tx];
      double Pm = 1.0;
#pragma unroll
      for (int m = 0; m < CH; ++m) {
        if (m < len) {
          Pm = Pm * __ldg(c_fwd + m * S);
          v[m] = v[m] + Pm * carry;
        }
      }
    }
    // back substitution, chunk-local with carry-in 0
    double x = 0.0, R = 1.0;
#pragma unroll
    for (int m = CH - 1; m >= 0; --m) {
      if (m < len) {
        const double b = __ldg(c_bwd + m * S);
        x = v[m] + b * x;
        R = R * b;
        v[m] = x;
      }
    }
    if (in_tile) {
      sX[c * TW + tx] = x;
      sR[c * TW + tx] = R;
    }
    __syncthreads();
    if (c < NC - 1 && len > 0) {
      double carry = 0.0;
      for (int cc = NC - 1; cc > c; --cc) carry = sR[cc * TW + tx] * carry + sX[cc * TW + tx];
      double Rm = 1.0;
#pragma unroll
      for (int m = CH - 1; m >= 0; --m) {
        if (m < len) {
          Rm = Rm * __ldg(c_bwd + m * S);
          v[m] = v[m] + Rm * carry;
        }
      }
    }
    if (AX == 2 && sources_after) {
      const int64_t vox0 = vcol / S + (int64_t)k0 * plane;  // voxel of the chunk's point 0
#pragma unroll
      for (int m = 0; m < CH; ++m) {
        if (m < len) {
          const int64_t vox = vox0 + m * plane;
          double x = v[m];
          if (a.bulk) {
            const int e = __ldg(a.bulk_map + vox);
            if (e >= 0)
              x = bulk_update(x, __ldg(a.bulk_st + (int64_t)e * S + s),
                              __ldg(a.bulk_su + (int64_t)e * S + s), a.dt);
          }
          if (a.cells) {
            const int r = __ldg(a.ag_map + vox);
            if (r >= 0) x = grid_cells(a, x, r, (uint64_t)vox, s);
          }
          ptr[m * ls] = x;
        }
      }
    } else {
#pragma unroll
      for (int m = 0; m < CH; ++m)
        if (m < len) ptr[m * ls] = v[m];
    }
    __syncthreads();  // the carries of this tile are read before the next overwrites them
  }
}

// nsteps whole steps with CH-point chunks (4 or 8: lines of <= 64 points in
// at most 16 or 8 chunks); launched cooperatively (every block resident) with
// 4 * blockDim.x doubles of dynamic shared memory.
template <int CH>
__global__ void __launch_bounds__(128) grid_steps_kernel(const GridStepArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double grid_carries[];
  const int first = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  const bool sources = a.bulk || a.cells;
  for (int step = 0; step < a.nsteps; ++step) {
    // the first step's sources get a phase of their own; later steps' were
    // applied as the previous z phase stored its lines
    if (sources && step == 0) {
      grid_sources(a, first, stride);
      grid.sync();
    }
    grid_axis<0, CH>(a, grid_carries);
    grid.sync();
    grid_axis<1, CH>(a, grid_carries);
    grid.sync();
    grid_axis<2, CH>(a, grid_carries, sources && step + 1 < a.nsteps);
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
