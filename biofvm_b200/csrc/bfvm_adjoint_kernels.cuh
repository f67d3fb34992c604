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

// Per-substrate sums over the field of a*(L_axis y) and a*y: block (S, W)
// threads, thread (s, w) walks voxels w, w + W*gridDim.x, ...; each block
// writes its partial sums to part[block][2S] (deterministic order).
static __global__ void adj_axis_dot_kernel(const double* __restrict__ a, const double* __restrict__ y,
                                    int nx, int ny, int nz, int S, int axis,
                                    double* __restrict__ part) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* sL = reinterpret_cast<double*>(smem_raw);  // [W][S]
  double* sI = sL + blockDim.x * blockDim.y;
  const int s = threadIdx.x, w = threadIdx.y, W = blockDim.y;
  const int64_t N = (int64_t)nx * ny * nz;
  const int64_t jump = axis == 0 ? 1 : (axis == 1 ? nx : (int64_t)nx * ny);
  const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
  double accL = 0.0, accI = 0.0;
  for (int64_t v = (int64_t)blockIdx.x * W + w; v < N; v += (int64_t)gridDim.x * W) {
    int k;
    if (axis == 0)
      k = (int)(v % nx);
    else if (axis == 1)
      k = (int)((v / nx) % ny);
    else
      k = (int)(v / ((int64_t)nx * ny));
    const int64_t q = v * S + s;
    const double yv = y[q];
    double ly = 0.0;
    if (k > 0) ly += yv - y[q - jump * S];
    if (k < n - 1) ly += yv - y[q + jump * S];
    const double av = a[q];
    accL += av * ly;
    accI += av * yv;
  }
  sL[w * S + s] = accL;
  sI[w * S + s] = accI;
  __syncthreads();
  if (w == 0) {
    double L = 0.0, I = 0.0;
    for (int u = 0; u < W; ++u) {
      L += sL[u * S + s];
      I += sI[u * S + s];
    }
    part[(int64_t)blockIdx.x * 2 * S + s] = L;
    part[(int64_t)blockIdx.x * 2 * S + S + s] = I;
  }
}

// acc[2S] -= sum over blocks of part (in block order): the solve's
// contributions -a.(L y) and -a.y.
static __global__ void adj_reduce_parts_kernel(const double* __restrict__ part, int blocks, int S,
                                        double* __restrict__ acc) {
  const int t = threadIdx.x;
  if (t >= 2 * S) return;
  double sum = 0.0;
  for (int b = 0; b < blocks; ++b) sum += part[(int64_t)b * 2 * S + t];
  acc[t] -= sum;
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
