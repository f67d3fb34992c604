// Device kernels of the B200 transport path.
//
// Density field: one array [nz][ny][nx][S] (substrate innermost), the
// reference's logical [voxel][substrate] order made contiguous.
//
// LOD sweep (BioFVM_solvers.cpp:175-273).  Along one axis every (line,
// substrate) pair is an independent tridiagonal system solved by the Thomas
// algorithm with precomputed coefficients:
//   forward   q_0 = p_0/d_0,  q_k = (p_k + c1*q_{k-1})/d_k     (:186-194)
//   backward  x_{n-1} = q_{n-1},  x_k = q_k - cx_k*x_{k+1}       (:196-200)
// Both are first-order linear recurrences, so a line is cut into chunks of
// CH points, one chunk per thread, held in registers:
//   1. each thread runs the recurrence over its chunk with carry-in 0 and
//      records the chunk's transfer (end value, product of slopes);
//   2. the transfers of the chunks of one line are folded through shared
//      memory to give every chunk its true carry-in;
//   3. each thread corrects its chunk: value += (running slope product)*carry.
// Every density element is read once and written once per sweep.
//
// A thread block is TW columns x NC chunks (blockDim = (TW, NC)); a
// "column" is one (line, substrate) pair and consecutive columns are
// consecutive addresses for the y and z sweeps, so every warp load/store is a
// contiguous TW*sizeof(T) run.  For the x sweep the S substrates of a row are
// the contiguous run.
//
// The x sweep also carries the rest of the step in its prologue: bulk
// sources/sinks, then cell sources/sinks (agents in reference order), then
// the Dirichlet overwrite; its epilogue is the Dirichlet overwrite that the
// reference does before the y sweep, and the y sweep's epilogue is the one
// before the z sweep.  These per-voxel updates use the same IEEE operations
// in the same order as the reference (no FMA contraction), so they are
// bit-exact; only the sweeps' rounding differs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bfvm {

enum : int {
  kFuseBulk = 1,
  kFuseCells = 2,
  kFuseDirPro = 4,   // Dirichlet before the sweep
  kFuseDirEpi = 8,   // Dirichlet after the sweep (= before the next axis)
};

// Coefficients of one axis, [n][S] each, in the sweep's precision.
template <typename T>
struct AxisCoef {
  const T* inv_den;  // 1 / thomas_denom
  const T* fwd;      // c1 / thomas_denom: slope of the forward recurrence
  const T* bwd;      // -thomas_c: slope of the back substitution
  const T* c1;       // [S] dt*D/dx^2
};

// Entries grouped by (line, chunk) segment: off[line*NC + c] .. off[+1].
// pos = point index along the line; a/b = per-substrate payload [E][S].
struct SegList {
  const int* off = nullptr;
  const int* pos = nullptr;
  const double* a = nullptr;
  const double* b = nullptr;
};

// T: the field's element type; CT: the type the sweep computes in (CT = T,
// or double over a float field).
template <typename T, typename CT = T>
struct SweepArgs {
  T* p;
  T* out;                // where the solved lines go (p: in place)
  int64_t col0;          // first column of this launch (a slab of planes)
  int64_t ncols;         // end of the launch's columns (all (line, substrate) columns)
  int64_t C;             // columns per outer block
  int64_t outer_stride;  // elements between outer blocks
  int64_t line_stride;   // elements between consecutive points of a line
  int n;                 // points per line
  int nchunks;           // NC = ceil(n / CH)
  int S;
  AxisCoef<CT> coef;
  SegList bulk, cells, dir_pro, dir_epi;
  double dt;
  int fuse;
};

template <typename T, int CH>
__device__ __forceinline__ T reg_get(const T (&v)[CH], int m) {
  T r = v[0];
#pragma unroll
  for (int q = 1; q < CH; ++q) r = (q == m) ? v[q] : r;
  return r;
}

template <typename T, int CH>
__device__ __forceinline__ void reg_set(T (&v)[CH], int m, T x) {
#pragma unroll
  for (int q = 0; q < CH; ++q) v[q] = (q == m) ? x : v[q];
}

// Bulk update of one voxel-substrate (BioFVM_microenvironment.cpp:603-609):
// p += dt*(S*T); p /= (U+S)*dt + 1.  st = S*T and su = U+S are stored.
__device__ __forceinline__ double bulk_update(double x, double st, double su, double dt) {
  x = __dadd_rn(x, __dmul_rn(dt, st));
  return __ddiv_rn(x, __dadd_rn(__dmul_rn(su, dt), 1.0));
}

// One agent's update (BioFVM_basic_agent.cpp:234-235): p += temp1; p /= temp2.
__device__ __forceinline__ double cell_update(double x, double t1, double t2) {
  return __ddiv_rn(__dadd_rn(x, t1), t2);
}

template <typename T, int CH>
__device__ __forceinline__ void apply_dirichlet_seg(T (&v)[CH], const SegList& L, int64_t seg,
                                                    int k0, int S, int s) {
  const int e0 = __ldg(L.off + seg), e1 = __ldg(L.off + seg + 1);
  for (int e = e0; e < e1; ++e) {
    const int m = __ldg(L.pos + e) - k0;
    reg_set<T, CH>(v, m, (T)__ldg(L.a + (int64_t)e * S + s));
  }
}

// MODE selects the fused work: kSweepPlain (z), kSweepDirEpi (y: Dirichlet
// after the sweep), kSweepFull (x: bulk/cells/Dirichlet prologue + Dirichlet
// epilogue, each switched by SweepArgs::fuse).  Separate instantiations keep
// the plain sweeps free of the prologue's registers.
enum : int { kSweepPlain = 0, kSweepDirEpi = 1, kSweepFull = 2 };

// MINB = minimum resident blocks per SM requested from the compiler (1 or 2):
// 2 caps registers at 64 per thread so two 512-thread blocks fit an SM.
// Largest block of lod_sweep_kernel for a chunk length: 32-point chunks keep
// 256 threads so that each thread has the registers for its chunk.
constexpr int sweep_max_threads(int ch) { return ch >= 32 ? 256 : 512; }

template <typename T, int CH, int MODE, int MINB, typename CT = T>
__global__ void __launch_bounds__(sweep_max_threads(CH), MINB)
    lod_sweep_kernel(const SweepArgs<T, CT> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int TW = blockDim.x;
  const int NC = blockDim.y;
  CT* sQ = reinterpret_cast<CT*>(smem_raw);  // [NC][TW] forward chunk end values
  CT* sP = sQ + NC * TW;                    // forward chunk slope products
  CT* sX = sP + NC * TW;                    // backward chunk start values
  CT* sR = sX + NC * TW;                    // backward chunk slope products

  const int tx = threadIdx.x;
  const int c = threadIdx.y;
  const int64_t vcol = a.col0 + (int64_t)blockIdx.x * TW + tx;
  const bool active = vcol < a.ncols;
  const int S = a.S;
  const int k0 = c * CH;
  // points of this chunk that exist (partial last chunk, empty chunks)
  const int len = active ? max(0, min(CH, a.n - k0)) : 0;

  T* ptr = a.p;
  int s = 0;
  int64_t seg = 0;
  if (active) {
    const int64_t outer = vcol / a.C;
    const int64_t col = vcol - outer * a.C;
    ptr = a.p + outer * a.outer_stride + col + (int64_t)k0 * a.line_stride;
    s = (int)(col % S);
    seg = (vcol / S) * a.nchunks + c;
  }
  const int64_t ls = a.line_stride;

  CT v[CH];
#pragma unroll
  for (int m = 0; m < CH; ++m) v[m] = (m < len) ? (CT)ptr[m * ls] : CT(0);

  if (MODE == kSweepFull && active) {
    if (a.fuse & kFuseBulk) {
      const int e0 = __ldg(a.bulk.off + seg), e1 = __ldg(a.bulk.off + seg + 1);
      for (int e = e0; e < e1; ++e) {
        const int m = __ldg(a.bulk.pos + e) - k0;
        const int64_t q = (int64_t)e * S + s;
        double x = (double)reg_get<CT, CH>(v, m);
        x = bulk_update(x, __ldg(a.bulk.a + q), __ldg(a.bulk.b + q), a.dt);
        reg_set<CT, CH>(v, m, (CT)x);
      }
    }
    if (a.fuse & kFuseCells) {
      // Agents of this chunk sorted by (voxel, list order): applying them in
      // sequence keeps the reference's order for agents sharing a voxel.
      // Consecutive agents of one voxel accumulate in FP64 before rounding.
      const int e0 = __ldg(a.cells.off + seg), e1 = __ldg(a.cells.off + seg + 1);
      int e = e0;
      while (e < e1) {
        const int pos = __ldg(a.cells.pos + e);
        const int m = pos - k0;
        double x = (double)reg_get<CT, CH>(v, m);
        do {
          const int64_t q = (int64_t)e * S + s;
          x = cell_update(x, __ldg(a.cells.a + q), __ldg(a.cells.b + q));
          ++e;
        } while (e < e1 && __ldg(a.cells.pos + e) == pos);
        reg_set<CT, CH>(v, m, (CT)x);
      }
    }
    if (a.fuse & kFuseDirPro) apply_dirichlet_seg<CT, CH>(v, a.dir_pro, seg, k0, S, s);
  }

  // Coefficient rows of this chunk: [k][S] tables, stride S along the line.
  const CT* c_inv = a.coef.inv_den + (int64_t)k0 * S + s;
  const CT* c_fwd = a.coef.fwd + (int64_t)k0 * S + s;
  const CT* c_bwd = a.coef.bwd + (int64_t)k0 * S + s;

  // ---- forward elimination, chunk-local with carry-in 0 ----
  const CT c1 = active ? __ldg(a.coef.c1 + s) : CT(0);
  CT q = CT(0), P = CT(1);
#pragma unroll
  for (int m = 0; m < CH; ++m) {
    if (m < len) {
      q = (v[m] + c1 * q) * __ldg(c_inv + m * S);
      P = P * __ldg(c_fwd + m * S);
      v[m] = q;
    }
  }
  sQ[c * TW + tx] = q;
  sP[c * TW + tx] = P;
  __syncthreads();
  if (c > 0 && len > 0) {
    CT carry = CT(0);
    for (int cc = 0; cc < c; ++cc) carry = sP[cc * TW + tx] * carry + sQ[cc * TW + tx];
    CT Pm = CT(1);
#pragma unroll
    for (int m = 0; m < CH; ++m) {
      if (m < len) {
        Pm = Pm * __ldg(c_fwd + m * S);
        v[m] = v[m] + Pm * carry;
      }
    }
  }

  // ---- back substitution, chunk-local with carry-in 0 ----
  CT x = CT(0), R = CT(1);
#pragma unroll
  for (int m = CH - 1; m >= 0; --m) {
    if (m < len) {
      const CT b = __ldg(c_bwd + m * S);
      x = v[m] + b * x;
      R = R * b;
      v[m] = x;
    }
  }
  sX[c * TW + tx] = x;
  sR[c * TW + tx] = R;
  __syncthreads();
  if (c < NC - 1 && len > 0) {
    CT carry = CT(0);
    for (int cc = NC - 1; cc > c; --cc) carry = sR[cc * TW + tx] * carry + sX[cc * TW + tx];
    CT Rm = CT(1);
#pragma unroll
    for (int m = CH - 1; m >= 0; --m) {
      if (m < len) {
        Rm = Rm * __ldg(c_bwd + m * S);
        v[m] = v[m] + Rm * carry;
      }
    }
  }

  if (MODE != kSweepPlain && active && (a.fuse & kFuseDirEpi))
    apply_dirichlet_seg<CT, CH>(v, a.dir_epi, seg, k0, S, s);

  T* dst = a.out + (ptr - a.p);
#pragma unroll
  for (int m = 0; m < CH; ++m)
    if (m < len) dst[m * ls] = (T)v[m];
}

// ---------------------------------------------------------------------------
// Stand-alone per-voxel kernels (the individual simulate_* / apply_* calls).

// simulate_bulk_sources_and_sinks over the stored (non-identity) voxels.
template <typename T>
__global__ void bulk_kernel(T* __restrict__ p, int S, int64_t E, const int64_t* __restrict__ voxel,
                            const double* __restrict__ st, const double* __restrict__ su,
                            double dt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  const int64_t q = voxel[e] * S + s;
  p[q] = (T)bulk_update((double)p[q], st[t], su[t], dt);
}

// The same update with the coefficient rows shared between voxels: voxel
// e's (S*T, U+S) for density s are tab[(row[e]*S + s)*2 + {0,1}] (the table
// is small and stays in L1), so the stream is the density itself plus 8 B
// per listed voxel.
template <typename T>
__global__ void bulk_rows_kernel(T* __restrict__ p, int S, int64_t E,
                                 const int* __restrict__ voxel, const int* __restrict__ row,
                                 const double* __restrict__ tab, double dt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  const int64_t q = (int64_t)__ldg(voxel + e) * S + s;
  const double* c = tab + ((int64_t)__ldg(row + e) * S + s) * 2;
  p[q] = (T)bulk_update((double)p[q], __ldg(c), __ldg(c + 1), dt);
}

// simulate_cell_sources_and_sinks over the agents sorted by voxel (key[r] =
// voxel of the r-th sorted agent, idx[r] = its position in the agent list;
// the sort is stable).  One thread per (sorted agent, substrate): the thread
// of the first agent of each voxel applies all agents of that voxel in list
// order, the others return.  t1/t2 are [A][S] in list order.
template <typename T>
__global__ void cells_kernel(T* __restrict__ p, int S, int64_t A, const uint64_t* __restrict__ key,
                             const int* __restrict__ idx, const double* __restrict__ t1,
                             const double* __restrict__ t2) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A * S) return;
  const int64_t r = t / S;
  const int s = (int)(t - r * S);
  const uint64_t v = key[r];
  if (r > 0 && key[r - 1] == v) return;
  const int64_t q = (int64_t)v * S + s;
  double x = (double)p[q];
  for (int64_t e = r; e < A && key[e] == v; ++e) {
    const int64_t a = idx[e];
    x = cell_update(x, t1[a * S + s], t2[a * S + s]);
  }
  p[q] = (T)x;
}

static __global__ void iota_kernel(int* __restrict__ out, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (int)t;
}

// a[r][col] = v for r < rows (row pitch `pitch` elements)
static __global__ void fill_column_kernel(double* __restrict__ a, int64_t rows, int pitch, int col,
                                   double v) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < rows) a[t * pitch + col] = v;
}

// apply_dirichlet_conditions over the de-duplicated node list.
template <typename T>
__global__ void dirichlet_kernel(T* __restrict__ p, int S, int64_t E, const int64_t* __restrict__ voxel,
                                 const double* __restrict__ val) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  p[voxel[e] * S + s] = (T)val[t];
}

// out[e][s] = p[voxel[e]][s]
template <typename T>
__global__ void gather_kernel(const T* __restrict__ p, int S, int64_t E, const int64_t* __restrict__ voxel,
                              double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  out[t] = (double)p[voxel[e] * S + s];
}

// p[voxel[e]][s] = in[e][s]
template <typename T>
__global__ void scatter_kernel(T* __restrict__ p, int S, int64_t E, const int64_t* __restrict__ voxel,
                               const double* __restrict__ in) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * S) return;
  const int64_t e = t / S;
  const int s = (int)(t - e * S);
  p[voxel[e] * S + s] = (T)in[t];
}

// Microenvironment::compute_all_gradient_vectors (BioFVM_microenvironment.cpp:
// 702-787): central differences along each axis at the points with a
// neighbour on both sides, g = (p[n + jump] - p[n - jump]) / (2 d); the
// components of points at an axis end are left as they are.  g is
// [N][S][3] FP64.
template <typename T>
__global__ void gradient_kernel(const T* __restrict__ p, int nx, int ny, int nz, int S,
                                double two_dx, double two_dy, double two_dz,
                                double* __restrict__ g) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t NS = (int64_t)nx * ny * nz * S;
  if (t >= NS) return;
  const int64_t n = t / S;
  const int i = (int)(n % nx);
  const int j = (int)((n / nx) % ny);
  const int k = (int)(n / ((int64_t)nx * ny));
  const int64_t jx = S, jy = (int64_t)nx * S, jz = (int64_t)nx * ny * S;
  double* out = g + 3 * t;
  if (i > 0 && i < nx - 1)
    out[0] = __ddiv_rn(__dsub_rn((double)p[t + jx], (double)p[t - jx]), two_dx);
  if (j > 0 && j < ny - 1)
    out[1] = __ddiv_rn(__dsub_rn((double)p[t + jy], (double)p[t - jy]), two_dy);
  if (k > 0 && k < nz - 1)
    out[2] = __ddiv_rn(__dsub_rn((double)p[t + jz], (double)p[t - jz]), two_dz);
}

// The same central differences with the grid laid over the mesh: block
// (bx, j, k) covers 256 consecutive (i, s) elements of row (j, k), so a thread
// finds its point with one 32-bit division by S instead of 64-bit divisions
// of a flat index (rows: gridDim.y = ny, gridDim.z = nz).
// The block's 256 x 3 results are staged in shared memory and written back
// as contiguous runs (components at an axis end keep their old value, read
// back only there).  Blocks of 256 threads.
template <typename T>
__global__ void __launch_bounds__(256) gradient_rows_kernel(
    const T* __restrict__ p, int nx, int ny, int nz, int S, double two_dx, double two_dy,
    double two_dz, double* __restrict__ g) {
  __shared__ double buf[3 * 256];
  const int e0 = blockIdx.x * 256;
  const int e = e0 + threadIdx.x;  // (i, s) within the row
  const int count = min(256, nx * S - e0);
  const int j = blockIdx.y, k = blockIdx.z;
  const int64_t row0 = ((int64_t)k * ny + j) * nx * S;  // first element of the row
  if (threadIdx.x < count) {
    const int i = e / S;
    const int64_t t = row0 + e;
    const int64_t jx = S, jy = (int64_t)nx * S, jz = (int64_t)nx * ny * S;
    double* b = buf + 3 * threadIdx.x;
    b[0] = (i > 0 && i < nx - 1)
               ? __ddiv_rn(__dsub_rn((double)p[t + jx], (double)p[t - jx]), two_dx)
               : g[3 * t];
    b[1] = (j > 0 && j < ny - 1)
               ? __ddiv_rn(__dsub_rn((double)p[t + jy], (double)p[t - jy]), two_dy)
               : g[3 * t + 1];
    b[2] = (k > 0 && k < nz - 1)
               ? __ddiv_rn(__dsub_rn((double)p[t + jz], (double)p[t - jz]), two_dz)
               : g[3 * t + 2];
  }
  __syncthreads();
  double* out = g + 3 * (row0 + e0);
  for (int c = threadIdx.x; c < 3 * count; c += 256) out[c] = buf[c];
}

// Lines longer than the chunked kernels take (more than 1024 points): one
// thread per (line, density) column runs the reference's Thomas sequence
// (BioFVM_solvers.cpp:186-200: p_0 /= d_0; p_k = (p_k + c1 p_{k-1}) / d_k;
// then p_k -= cx_k p_{k+1}), each operation rounded on its own, so the
// result equals the reference's for an FP64 field.  Consecutive columns are
// consecutive addresses for the y and z axes (the S densities of consecutive
// rows for x).  The forward values are stored and read back by the backward
// pass: two reads and two writes per element.  den, cx: [n][S]; c1: [S].
template <typename T>
__global__ void long_line_kernel(T* __restrict__ p, T* __restrict__ out, int64_t col0,
                                 int64_t ncols, int64_t C, int64_t outer_stride,
                                 int64_t line_stride, int n, int S,
                                 const double* __restrict__ den, const double* __restrict__ cx,
                                 const double* __restrict__ c1v) {
  const int64_t vcol = col0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (vcol >= ncols) return;
  const int64_t outer = vcol / C;
  const int64_t col = vcol - outer * C;
  const int s = (int)(col % S);
  const int64_t off = outer * outer_stride + col;
  const T* q = p + off;
  T* o = out + off;
  const double c1 = __ldg(c1v + s);
  double prev = __ddiv_rn((double)q[0], __ldg(den + s));
  o[0] = (T)prev;
  for (int k = 1; k < n; ++k) {
    prev = __ddiv_rn(__dadd_rn((double)q[k * line_stride], __dmul_rn(c1, prev)),
                     __ldg(den + (int64_t)k * S + s));
    o[k * line_stride] = (T)prev;
  }
  double next = prev;
  for (int k = n - 2; k >= 0; --k) {
    next = __dsub_rn((double)o[k * line_stride], __dmul_rn(__ldg(cx + (int64_t)k * S + s), next));
    o[k * line_stride] = (T)next;
  }
}

// Joins the z slabs of a field split by planes over several solvers, after
// each slab's z sweep ran with zero carries at its ends (x').  One thread
// per (i, j, density) column of this slab.  planes [R][2][C]: every slab's
// first and last local plane after its sweep (C = nx*ny*S values each);
// cst [R][S][3] {P, Gs, R} per slab; pt [nz][S][2] {G, Rk} of this slab's
// planes.  The forward value entering slab r folds the slabs before it
// (Q = P Q + last), the solution on the first plane after this slab folds
// the slabs after it from the far end (X = first + C Gs + R X); then
// x_k = x'_k + C G_k + X Rk_k on every plane of this slab.
template <int MAXR>
__global__ void zslab_fixup_kernel(double* __restrict__ p, int64_t C, int S, int nz, int R,
                                   int rank, const double* __restrict__ planes,
                                   const double* __restrict__ cst,
                                   const double* __restrict__ pt) {
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= C) return;
  const int s = (int)(col % S);
  double carry_in[MAXR];
  double Q = 0.0;
#pragma unroll
  for (int r = 0; r < MAXR; ++r) {
    if (r < R) {
      carry_in[r] = Q;
      Q = __ldg(cst + ((int64_t)r * S + s) * 3) * Q + __ldg(planes + ((int64_t)r * 2 + 1) * C + col);
    }
  }
  double X = 0.0;
#pragma unroll
  for (int r = MAXR - 1; r >= 0; --r) {
    if (r < R && r > rank) {
      const double* k = cst + ((int64_t)r * S + s) * 3;
      X = __ldg(planes + (int64_t)r * 2 * C + col) + carry_in[r] * __ldg(k + 1) + __ldg(k + 2) * X;
    }
  }
  double Cr = 0.0;
#pragma unroll
  for (int r = 0; r < MAXR; ++r)
    if (r == rank) Cr = carry_in[r];
  for (int k = 0; k < nz; ++k) {
    const double* g = pt + ((int64_t)k * S + s) * 2;
    double* q = p + (int64_t)k * C + col;
    *q = *q + Cr * __ldg(g) + X * __ldg(g + 1);
  }
}

template <typename Dst, typename Src>
__global__ void convert_kernel(Dst* __restrict__ dst, const Src* __restrict__ src, int64_t count) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) dst[t] = (Dst)src[t];
}

}  // namespace bfvm
