// Kernels that advance many independent microenvironments in one launch.
//
// Every instance keeps its own density field, Thomas tables, bulk list,
// agents and Dirichlet nodes (the state of one bfvm_solver).  A launch covers
// the instances of one group: its work is the concatenation of the
// instances' work, and each thread block (sweeps) or thread (per-voxel
// updates) finds its instance by a binary search over the instances' first
// work index.  The arithmetic is that of the single-instance kernels in
// bfvm_kernels.cuh, operation for operation.
#pragma once

#include "bfvm_kernels.cuh"

namespace bfvm {

// Index of the last entry whose first work index is <= w (first[0] == 0).
template <typename D>
__device__ __forceinline__ int find_owner(const D* __restrict__ d, int count, int64_t w) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&d[mid].first) <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The lines of one instance along one axis.  A work item is `tw` consecutive
// columns x all chunks of their lines; tw * nchunks <= blockDim.x.
template <typename T>
struct BatchSweep {
  T* p;
  AxisCoef<T> coef;
  int64_t ncols;         // (line, substrate) columns
  int64_t C;             // columns per outer block
  int64_t outer_stride;  // elements between outer blocks
  int64_t line_stride;   // elements between consecutive points of a line
  int64_t first;         // first work item of this instance in the launch
  int n, nchunks, S, tw;
};

// Largest block of the batched sweep for a chunk length: 32 points per
// thread need the registers of a 256-thread block.
constexpr int batch_max_threads(int ch) { return ch >= 32 ? 256 : 512; }

// LOD sweep of many instances (BioFVM_solvers.cpp:175-273, one axis): the
// chunked Thomas recurrence of lod_sweep_kernel, one work item per block.
template <typename T, int CH>
__global__ void __launch_bounds__(batch_max_threads(CH)) lod_batch_sweep_kernel(const BatchSweep<T>* __restrict__ sw,
                                                              int count) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nthreads = blockDim.x;
  T* sQ = reinterpret_cast<T*>(smem_raw);  // [NC][TW] forward chunk end values
  T* sP = sQ + nthreads;                   // forward chunk slope products
  T* sX = sP + nthreads;                   // backward chunk start values
  T* sR = sX + nthreads;                   // backward chunk slope products

  const int64_t item = blockIdx.x;
  const BatchSweep<T>& d = sw[find_owner(sw, count, item)];
  const int TW = d.tw, NC = d.nchunks, S = d.S, n = d.n;
  const int tid = threadIdx.x;
  const int c = tid / TW;
  const int tx = tid - c * TW;
  const int64_t vcol = (item - d.first) * TW + tx;
  const bool active = c < NC && vcol < d.ncols;
  const int k0 = c * CH;
  const int len = active ? max(0, min(CH, n - k0)) : 0;

  T* ptr = d.p;
  int s = 0;
  if (active) {
    const int64_t outer = vcol / d.C;
    const int64_t col = vcol - outer * d.C;
    ptr = d.p + outer * d.outer_stride + col + (int64_t)k0 * d.line_stride;
    s = (int)(col % S);
  }
  const int64_t ls = d.line_stride;

  T v[CH];
#pragma unroll
  for (int m = 0; m < CH; ++m) v[m] = (m < len) ? ptr[m * ls] : T(0);

  const T* c_inv = d.coef.inv_den + (int64_t)k0 * S + s;
  const T* c_fwd = d.coef.fwd + (int64_t)k0 * S + s;
  const T* c_bwd = d.coef.bwd + (int64_t)k0 * S + s;

  // forward elimination, chunk-local with carry-in 0
  const T c1 = active ? __ldg(d.coef.c1 + s) : T(0);
  T q = T(0), P = T(1);
#pragma unroll
  for (int m = 0; m < CH; ++m) {
    if (m < len) {
      q = (v[m] + c1 * q) * __ldg(c_inv + m * S);
      P = P * __ldg(c_fwd + m * S);
      v[m] = q;
    }
  }
  if (c < NC) {
    sQ[c * TW + tx] = q;
    sP[c * TW + tx] = P;
  }
  __syncthreads();
  if (c > 0 && len > 0) {
    T carry = T(0);
    for (int cc = 0; cc < c; ++cc) carry = sP[cc * TW + tx] * carry + sQ[cc * TW + tx];
    T Pm = T(1);
#pragma unroll
    for (int m = 0; m < CH; ++m) {
      if (m < len) {
        Pm = Pm * __ldg(c_fwd + m * S);
        v[m] = v[m] + Pm * carry;
      }
    }
  }

  // back substitution, chunk-local with carry-in 0
  T x = T(0), R = T(1);
#pragma unroll
  for (int m = CH - 1; m >= 0; --m) {
    if (m < len) {
      const T b = __ldg(c_bwd + m * S);
      x = v[m] + b * x;
      R = R * b;
      v[m] = x;
    }
  }
  if (c < NC) {
    sX[c * TW + tx] = x;
    sR[c * TW + tx] = R;
  }
  __syncthreads();
  if (c < NC - 1 && len > 0) {
    T carry = T(0);
    for (int cc = NC - 1; cc > c; --cc) carry = sR[cc * TW + tx] * carry + sX[cc * TW + tx];
    T Rm = T(1);
#pragma unroll
    for (int m = CH - 1; m >= 0; --m) {
      if (m < len) {
        Rm = Rm * __ldg(c_bwd + m * S);
        v[m] = v[m] + Rm * carry;
      }
    }
  }

#pragma unroll
  for (int m = 0; m < CH; ++m)
    if (m < len) ptr[m * ls] = v[m];
}

// A per-voxel list of one instance: `count` entries x S substrates, work
// indices first .. first + count*S.  Bulk: vox, a = S*T, b = U+S.
// Dirichlet: vox, a = values.  Cells: key/idx = agents sorted by voxel,
// a/b = temp1/temp2 in list order.
template <typename T>
struct BatchList {
  T* p;
  const int64_t* vox;
  const uint64_t* key;
  const int* idx;
  const double* a;
  const double* b;
  int64_t count;
  int64_t first;
  int S;
};

template <typename T>
__global__ void batch_bulk_kernel(const BatchList<T>* __restrict__ L, int count, int64_t work,
                                  double dt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= work) return;
  const BatchList<T>& d = L[find_owner(L, count, t)];
  const int64_t w = t - d.first;
  const int64_t e = w / d.S;
  const int s = (int)(w - e * d.S);
  const int64_t q = __ldg(d.vox + e) * d.S + s;
  d.p[q] = (T)bulk_update((double)d.p[q], __ldg(d.a + w), __ldg(d.b + w), dt);
}

template <typename T>
__global__ void batch_cells_kernel(const BatchList<T>* __restrict__ L, int count, int64_t work) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= work) return;
  const BatchList<T>& d = L[find_owner(L, count, t)];
  const int S = d.S;
  const int64_t w = t - d.first;
  const int64_t r = w / S;
  const int s = (int)(w - r * S);
  const uint64_t v = __ldg(d.key + r);
  if (r > 0 && __ldg(d.key + r - 1) == v) return;
  const int64_t q = (int64_t)v * S + s;
  double x = (double)d.p[q];
  for (int64_t e = r; e < d.count && __ldg(d.key + e) == v; ++e) {
    const int64_t a = __ldg(d.idx + e);
    x = cell_update(x, __ldg(d.a + a * S + s), __ldg(d.b + a * S + s));
  }
  d.p[q] = (T)x;
}

template <typename T>
__global__ void batch_dirichlet_kernel(const BatchList<T>* __restrict__ L, int count,
                                       int64_t work) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= work) return;
  const BatchList<T>& d = L[find_owner(L, count, t)];
  const int64_t w = t - d.first;
  const int64_t e = w / d.S;
  const int s = (int)(w - e * d.S);
  d.p[__ldg(d.vox + e) * d.S + s] = (T)__ldg(d.a + w);
}

}  // namespace bfvm
