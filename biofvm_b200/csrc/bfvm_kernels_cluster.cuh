// Whole steps of a small microenvironment in one thread-block cluster.
//
// When the density field fits in the shared memory of a cluster (at most 8
// blocks of up to ~200 KB), one launch runs every step: block r of the
// cluster holds the z planes [r*pz, min(nz, (r+1)*pz)) of the field in its
// shared memory, applies the bulk, cell and Dirichlet updates of its planes,
// sweeps its x and y lines in place, and the z lines -- which cross every
// block -- are read from and written back to the blocks' shared memory
// through distributed shared memory.  Phases are separated by block and
// cluster barriers (hardware barriers that every thread of every block
// reaches the same number of times); nothing spins.  The field goes to and
// from global memory once per launch.
//
// Every line is solved with the reference's own operation sequence
// (BioFVM_solvers.cpp:186-200): p_0 /= d_0; p_i += c1 p_{i-1}, p_i /= d_i;
// p_i -= cx_i p_{i+1}, each multiply, add and divide rounded on its own (no
// fused multiply-add), so a step here equals the reference's FP64 step bit
// for bit.
#pragma once

#include <cooperative_groups.h>

#include "bfvm_kernels.cuh"

namespace bfvm {

struct ClusterStepArgs {
  double* p;  // [nz][ny][nx][S]
  int nx, ny, nz, S;
  int pz;  // z planes per block
  int nsteps;
  double dt;
  bool bulk, cells, diffusion;
  // Thomas coefficients per axis: den[n][S], cx[n][S], c1[S]
  const double* den[3];
  const double* cx[3];
  const double* c1[3];
  // bulk list (ascending voxels), S*T and U+S per (entry, substrate)
  int64_t nbulk;
  const int64_t* bulk_vox;
  const double* bulk_st;
  const double* bulk_su;
  // agents sorted by voxel (stable): key = voxel, idx = list position;
  // temp1/temp2 [A][S] in list order
  int64_t nagents;
  const uint64_t* ag_key;
  const int* ag_idx;
  const double* ag_t1;
  const double* ag_t2;
  // Dirichlet nodes (unique voxels, last value wins) and values [E][S]
  int64_t ndir;
  const int64_t* dir_vox;
  const double* dir_val;
  // per block (at most 8): its Dirichlet nodes [dir_lo, dir_hi) and bulk
  // entries [bulk_lo, bulk_hi) (both lists ascending in voxel); dir_staged:
  // the block's Dirichlet nodes are copied to its shared memory after the
  // field (values [n][S], then local voxel indices [n])
  int dir_lo[8], dir_hi[8];
  int64_t bulk_lo[8], bulk_hi[8];
  bool dir_staged;
};

// One line of n points in this block's shared memory (stride apart),
// solved in place with the reference's sequence.
__device__ __forceinline__ void cluster_line_smem(double* p, int64_t stride, int n,
                                                  const double* __restrict__ den,
                                                  const double* __restrict__ cx, double c1,
                                                  int S, int s) {
  double prev = __ddiv_rn(p[0], __ldg(den + s));
  p[0] = prev;
  for (int k = 1; k < n; ++k) {
    prev = __ddiv_rn(__dadd_rn(p[k * stride], __dmul_rn(c1, prev)),
                     __ldg(den + (int64_t)k * S + s));
    p[k * stride] = prev;
  }
  double next = prev;
  for (int k = n - 2; k >= 0; --k) {
    next = __dsub_rn(p[k * stride], __dmul_rn(__ldg(cx + (int64_t)k * S + s), next));
    p[k * stride] = next;
  }
}

// One line of n <= NMAX points spread over the cluster's blocks (a z line):
// gathered into registers with independent loads, solved there with the
// reference's sequence, scattered back.  at(k) is the address of point k.
template <int NMAX, typename At>
__device__ __forceinline__ void cluster_line_regs(At at, int n, const double* __restrict__ den,
                                                  const double* __restrict__ cx, double c1,
                                                  int S, int s) {
  double v[NMAX];
#pragma unroll
  for (int k = 0; k < NMAX; ++k)
    if (k < n) v[k] = *at(k);
  double prev = __ddiv_rn(v[0], __ldg(den + s));
  v[0] = prev;
#pragma unroll
  for (int k = 1; k < NMAX; ++k)
    if (k < n) {
      prev = __ddiv_rn(__dadd_rn(v[k], __dmul_rn(c1, prev)), __ldg(den + (int64_t)k * S + s));
      v[k] = prev;
    }
  double next = prev;  // v[n-1]
#pragma unroll
  for (int k = NMAX - 2; k >= 0; --k)
    if (k < n - 1) {
      next = __dsub_rn(v[k], __dmul_rn(__ldg(cx + (int64_t)k * S + s), next));
      v[k] = next;
    }
#pragma unroll
  for (int k = 0; k < NMAX; ++k)
    if (k < n) *at(k) = v[k];
}

template <int NMAX>
__global__ void __launch_bounds__(256, 1) cluster_steps_kernel(const ClusterStepArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) double slab[];  // [pz][ny][nx][S] of this block
  const int rank = (int)cluster.block_rank();
  const int nblocks = (int)cluster.num_blocks();
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nx = a.nx, ny = a.ny, nz = a.nz, S = a.S;
  const int z0 = min(nz, rank * a.pz), z1 = min(nz, z0 + a.pz), nzr = z1 - z0;
  const int64_t plane = (int64_t)nx * ny;          // voxels per z plane
  const int64_t mine = (int64_t)nzr * plane * S;   // elements held here
  const int64_t first = (int64_t)z0 * plane;       // first voxel held here
  double* g = a.p + first * S;

  for (int64_t i = tid; i < mine; i += nt) slab[i] = g[i];
  // local index of a voxel of this block's planes, or -1
  auto local = [&](int64_t v) -> int64_t {
    const int64_t lv = v - first;
    return (lv >= 0 && lv < (int64_t)nzr * plane) ? lv : -1;
  };
  // this block's Dirichlet nodes, staged in shared memory when they fit
  const int d0 = a.dir_lo[rank], nd = a.dir_hi[rank] - d0;
  double* sdv = slab + (int64_t)a.pz * plane * S;  // [nd][S]
  int* sdi = reinterpret_cast<int*>(sdv + (a.dir_staged ? (int64_t)nd * S : 0));  // [nd]
  if (a.dir_staged) {
    for (int64_t w = tid; w < (int64_t)nd * S; w += nt) sdv[w] = __ldg(a.dir_val + (int64_t)d0 * S + w);
    for (int e = tid; e < nd; e += nt) sdi[e] = (int)(__ldg(a.dir_vox + d0 + e) - first);
  }
  auto dirichlet = [&]() {
    for (int64_t w = tid; w < (int64_t)nd * S; w += nt) {
      const int64_t e = w / S;
      const int s = (int)(w - e * S);
      if (a.dir_staged)
        slab[(int64_t)sdi[e] * S + s] = sdv[w];
      else
        slab[(__ldg(a.dir_vox + d0 + e) - first) * S + s] =
            __ldg(a.dir_val + (int64_t)(d0 + e) * S + s);
    }
  };
  // this block's agents: the sorted keys in [first, first + nzr*plane)
  __shared__ int64_t ag_range[2];
  if (tid < 2) {
    const uint64_t want = (uint64_t)(first + (tid ? (int64_t)nzr * plane : 0));
    int64_t lo = 0, hi = a.nagents;  // first key >= want
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (__ldg(a.ag_key + mid) < want)
        lo = mid + 1;
      else
        hi = mid;
    }
    ag_range[tid] = lo;
  }
  cluster.sync();
  const int64_t a0 = ag_range[0], a1 = ag_range[1];

  for (int step = 0; step < a.nsteps; ++step) {
    // bulk -> cells (BioFVM_microenvironment.cpp:603-609, BioFVM_basic_agent.cpp:234-235)
    if (a.bulk)
      for (int64_t w = a.bulk_lo[rank] * S + tid; w < a.bulk_hi[rank] * S; w += nt) {
        const int64_t e = w / S;
        const int s = (int)(w - e * S);
        double* q = slab + (__ldg(a.bulk_vox + e) - first) * S + s;
        *q = bulk_update(*q, __ldg(a.bulk_st + w), __ldg(a.bulk_su + w), a.dt);
      }
    __syncthreads();
    if (a.cells)
      for (int64_t w = a0 * S + tid; w < a1 * S; w += nt) {
        const int64_t r = w / S;
        const int s = (int)(w - r * S);
        const uint64_t v = __ldg(a.ag_key + r);
        if (r > a0 && __ldg(a.ag_key + r - 1) == v) continue;
        const int64_t lv = local((int64_t)v);
        if (lv < 0) continue;
        double x = slab[lv * S + s];
        for (int64_t e = r; e < a1 && __ldg(a.ag_key + e) == v; ++e) {
          const int64_t ai = __ldg(a.ag_idx + e);
          x = cell_update(x, __ldg(a.ag_t1 + ai * S + s), __ldg(a.ag_t2 + ai * S + s));
        }
        slab[lv * S + s] = x;
      }
    __syncthreads();
    if (a.diffusion) {
      // x lines of this block's planes (BioFVM_solvers.cpp:177-204)
      dirichlet();
      __syncthreads();
      for (int64_t l = tid; l < (int64_t)nzr * ny * S; l += nt) {
        const int s = (int)(l % S);
        const int64_t row = l / S;  // (local plane, j)
        cluster_line_smem(slab + row * nx * S + s, S, nx, a.den[0], a.cx[0],
                          __ldg(a.c1[0] + s), S, s);
      }
      __syncthreads();
      // y lines (:207-238)
      dirichlet();
      __syncthreads();
      for (int64_t l = tid; l < (int64_t)nzr * nx * S; l += nt) {
        const int s = (int)(l % S);
        const int64_t col = l / S;  // (local plane, i)
        const int64_t kl = col / nx, i = col - kl * nx;
        cluster_line_smem(slab + (kl * plane + i) * S + s, (int64_t)nx * S, ny, a.den[1],
                          a.cx[1], __ldg(a.c1[1] + s), S, s);
      }
      __syncthreads();
      // z lines cross every block: through distributed shared memory (:241-273)
      dirichlet();
      cluster.sync();
      for (int64_t l = (int64_t)rank * nt + tid; l < plane * S; l += (int64_t)nblocks * nt) {
        const int s = (int)(l % S);
        const int64_t ij = l / S;  // voxel within a plane
        cluster_line_regs<NMAX>(
            [&](int k) {
              const int owner = k / a.pz;
              double* remote = cluster.map_shared_rank(slab, owner);
              return remote + ((int64_t)(k - owner * a.pz) * plane + ij) * S + s;
            },
            nz, a.den[2], a.cx[2], __ldg(a.c1[2] + s), S, s);
      }
    }
    cluster.sync();
  }
  for (int64_t i = tid; i < mine; i += nt) g[i] = slab[i];
}

}  // namespace bfvm
