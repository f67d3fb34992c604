// Kernels of the adjoint (reverse-mode derivative) of the transport step.
//
// One forward step (FP64) is  p1 = bulk(p0);  p2 = cells(p1);
// p3 = D(p2), y_x = A_x^-1 p3;  p5 = D(y_x), y_y = A_y^-1 p5;
// p7 = D(y_y), y_z = A_z^-1 p7  (BioFVM_solvers.cpp:175-273), where D
// overwrites the Dirichlet nodes and A_a = (1 + c2) I + c1 L_a with L_a the
// Neumann Laplacian along axis a (diagonal 2, 1 at the line ends, -1 off the
// diagonal; 0 for a one-point line), c1 = dt D / dx^2, c2 = dt decay / 3
// (BioFVM_solvers.cpp:105-142).  A_a is symmetric, so the adjoint of a solve
// is the same solve, and the derivative of the loss with respect to c1 (c2)
// through one solve y = A^-1 x is -abar . (L y)  (-abar . y), abar = A^-1 ybar.
#pragma once

#include "bfvm_kernels.cuh"

namespace bfvm {

// Per-substrate sums over the field of a*(L_axis y) and a*y.  Blocks take
// whole rows (fixed y, z: nx*S contiguous elements), block b the rows b,
// b + gridDim.x, ...; blockDim.x is a multiple of S, so thread t keeps one
// density s = t % S and steps through x = t / S, t / S + blockDim.x / S, ...
// of each row (coalesced; the row's position along y and z is found once per
// row, and along x by counting).  Each block adds its per-density partial
// sums to part[block][2S], which accumulates over every solve of a backward
// run (zeroed at its start, reduced once at its end); the order of every sum
// is fixed.
static __global__ void adj_axis_dot_kernel(const double* __restrict__ a,
                                           const double* __restrict__ y, int nx, int ny, int nz,
                                           int S, int axis, double* __restrict__ part) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sL = reinterpret_cast<double*>(smem_raw);  // [blockDim.x]
  double* sI = sL + blockDim.x;
  const int t = threadIdx.x, B = blockDim.x;
  const int s = t % S, xstep = B / S;
  const int64_t rows = (int64_t)ny * nz;
  const int64_t RS = (int64_t)nx * S;
  const int64_t jump = axis == 1 ? RS : (int64_t)ny * RS;  // y and z neighbours
  double accL = 0.0, accI = 0.0;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int64_t zz = r / ny;
    const int yy = (int)(r - zz * ny);
    const bool lo = axis == 1 ? yy > 0 : zz > 0;
    const bool hi = axis == 1 ? yy < ny - 1 : zz < nz - 1;
    const double* yr = y + r * RS;
    const double* ar = a + r * RS;
    for (int x = t / S; x < nx; x += xstep) {
      const int64_t c = (int64_t)x * S + s;
      const double yv = yr[c];
      double ly = 0.0;
      if (axis == 0) {
        if (x > 0) ly += yv - yr[c - S];
        if (x < nx - 1) ly += yv - yr[c + S];
      } else {
        if (lo) ly += yv - yr[c - jump];
        if (hi) ly += yv - yr[c + jump];
      }
      const double av = ar[c];
      accL += av * ly;
      accI += av * yv;
    }
  }
  sL[t] = accL;
  sI[t] = accI;
  __syncthreads();
  if (t < S) {
    double L = 0.0, I = 0.0;
    for (int u = t; u < B; u += S) {
      L += sL[u];
      I += sI[u];
    }
    part[(int64_t)blockIdx.x * 2 * S + t] += L;
    part[(int64_t)blockIdx.x * 2 * S + S + t] += I;
  }
}

// acc[j] -= sum over blocks of part[.][j], one block of kAdjReduceThreads
// per output j in [0, 2S) (thread i sums blocks i, i + kAdjReduceThreads, ...,
// then a fixed tree): the solves' contributions -a.(L y) and -a.y.
constexpr int kAdjReduceThreads = 256;
static __global__ void __launch_bounds__(kAdjReduceThreads)
    adj_reduce_parts_kernel(const double* __restrict__ part, int blocks, int S,
                            double* __restrict__ acc) {
  __shared__ double sm[kAdjReduceThreads];
  const int j = blockIdx.x, i = threadIdx.x;
  double sum = 0.0;
  for (int b = i; b < blocks; b += kAdjReduceThreads) sum += part[(int64_t)b * 2 * S + j];
  sm[i] = sum;
  __syncthreads();
  for (int w = kAdjReduceThreads / 2; w > 0; w >>= 1) {
    if (i < w) sm[i] += sm[i + w];
    __syncthreads();
  }
  if (i == 0) acc[j] -= sm[0];
}

// a = 0 at the Dirichlet nodes (the adjoint of the overwrite).
static __global__ void adj_zero_nodes_kernel(double* __restrict__ a, int S, int64_t E,
                                      const int64_t* __restrict__ voxel) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  a[voxel[e] * S + s] = 0.0;
}

// Adjoint of the bulk update p1 = (p0 + dt S T) / ((U + S) dt + 1): a /= the
// same denominator, on the listed voxels.
static __global__ void adj_bulk_kernel(double* __restrict__ a, int S, int64_t E,
                                const int64_t* __restrict__ voxel, const double* __restrict__ su,
                                double dt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  const int64_t q = voxel[e] * S + s;
  a[q] = __ddiv_rn(a[q], __dadd_rn(__dmul_rn(su[t], dt), 1.0));
}

// Adjoint of the cell updates of one voxel (agents in list order,
// x_j = (x_{j-1} + t1_j) / t2_j, BioFVM_basic_agent.cpp:234-235): the
// thread of the first sorted agent of a voxel recomputes the chain from the
// step input (after the bulk update when bulk ran), then walks it backwards:
//   gt1_j += g / t2_j,  gt2_j -= g x_j / t2_j,  g /= t2_j,
// recovering x_{j-1} = x_j t2_j - t1_j.  gt1/gt2 are [A][S] in list order.
static __global__ void adj_cells_kernel(double* __restrict__ a, const double* __restrict__ p_in, int S,
                                 int64_t A, const uint64_t* __restrict__ key,
                                 const int* __restrict__ idx, const double* __restrict__ t1,
                                 const double* __restrict__ t2, int64_t nbulk,
                                 const int64_t* __restrict__ bulk_vox,
                                 const double* __restrict__ bulk_st,
                                 const double* __restrict__ bulk_su, double dt,
                                 double* __restrict__ gt1, double* __restrict__ gt2) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A * S) return;
  const int64_t r = t / S;
  const int s = (int)(t - r * S);
  const uint64_t v = key[r];
  if (r > 0 && key[r - 1] == v) return;
  const int64_t q = (int64_t)v * S + s;
  double x = p_in[q];
  if (nbulk > 0) {  // bulk list sorted by voxel
    int64_t lo = 0, hi = nbulk - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((uint64_t)bulk_vox[mid] < v)
        lo = mid + 1;
      else
        hi = mid;
    }
    if ((uint64_t)bulk_vox[lo] == v)
      x = bulk_update(x, bulk_st[lo * S + s], bulk_su[lo * S + s], dt);
  }
  int64_t end = r;
  while (end < A && key[end] == v) {
    const int64_t i = idx[end];
    x = cell_update(x, t1[i * S + s], t2[i * S + s]);
    ++end;
  }
  double g = a[q];
  for (int64_t e = end - 1; e >= r; --e) {
    const int64_t i = idx[e];
    const double b1 = t1[i * S + s], b2 = t2[i * S + s];
    gt1[i * S + s] += g / b2;
    gt2[i * S + s] -= g * x / b2;
    g = g / b2;
    x = x * b2 - b1;
  }
  a[q] = g;
}

}  // namespace bfvm
