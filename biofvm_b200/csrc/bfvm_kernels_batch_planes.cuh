// Whole steps of a group of independent microenvironments in one persistent
// cooperative launch, plane form (BFVM_BATCH_PLANES of bfvm_batch).
//
// The sweeps of one step are paired so that a step crosses L2 twice instead
// of three times, and every line is solved whole by one thread from shared
// memory (no chunk fold, no per-point table of prefix products):
//
//   xy phase   work item = one xy plane (fixed z) of one member, or a subset
//              of its densities when the whole plane does not fit: the block
//              copies the plane into shared memory, applies the bulk
//              updates (BioFVM_microenvironment.cpp:603-609) and then the
//              agents' updates in list order (BioFVM_basic_agent.cpp:234-235),
//              gives the Dirichlet nodes of every x line their values
//              (BioFVM_solvers.cpp:177), solves the x lines (:186-200), gives
//              the nodes of every y line their values (:207), solves the y
//              lines (:217-234) and writes the plane back;
//   z phase    work item = a strip of columns (x, density) of one xz plane
//              (fixed y): the block copies the strip's nz rows into shared
//              memory, gives the nodes of every z line their values (:241),
//              solves the z lines (:252-271) and writes the strip back.
//
// The bulk and cell updates of an x line are applied by the thread that then
// solves it, to the staged line: the bulk list is cut into runs of
// consecutive voxels of one x line with bitwise-equal rates (built on the
// host), agents are found by per-line offsets into the sorted agent list
// (plane_agent_lines_kernel); bulk first, then the agents in list order.  The x, y and z orders of the reference are kept,
// with a Dirichlet overwrite before each sweep.
//
// A line is solved with the recurrences of the chunked kernels taken over
// the whole line (the per-point work of BioFVM_solvers.cpp:186-200 with the
// division replaced by the precomputed reciprocal):
//   forward   q_k = a_k q_{k-1} + p_k / d_k      (a_k = c1 / d_k = -cx_k, q_{-1} = 0)
//   backward  x_k = q_k + a_k x_{k+1}            (x_{n-1} = q_{n-1})
// with the {1/d_k, a_k} pairs of the chunked kernels' tables, interleaved
// [point][density] (one 16-byte load per point).  Each thread walks its line
// in shared memory, so the dependent chain of a point is one FMA.
//
// Blocks take work items from a per-phase counter (one atomic per item,
// fetched one item ahead), so blocks that drew small items take more of
// them.  Phases are separated by the grid-wide barriers of the cooperative
// launch.  The field moves through L2 only (ld/st.global.cg): a block reads
// planes that other SMs wrote before the barrier, and L1 is not coherent
// across SMs.
#pragma once

#include <cooperative_groups.h>

#include "bfvm_kernels_batch_steps.cuh"

namespace bfvm {

constexpr int kPlaneThreads = 512;
// Shared memory of the block (one per SM): the plane or strip being solved
// (kPlaneSmemDoubles doubles, 208 KB: a 128 x 128 plane of one density at
// its padded pitch fits) and the {1/d, a} pairs of its lines
// (kPlaneTabPairs, 16 KB).
constexpr int kPlaneSmemDoubles = 26624;
constexpr int kPlaneTabPairs = 1024;
constexpr int kPlaneLoadBatch = 16;   // stores in flight per thread while writing back

// floor(n / d) as umulhi(n, M) with M = udiv_magic(d) (M = 0 stands for
// d = 1).  With M = floor((2^32 - 1) / d) + 1, M*d = 2^32 + e with 0 <= e < d,
// so n*M / 2^32 = n/d + n*e / (d*2^32) and the floor is exact whenever
// n*d <= 2^32; every use below has n and d under 2^16.
__host__ __device__ __forceinline__ uint32_t udiv_magic(uint32_t d) {
  return d == 1u ? 0u : 0xFFFFFFFFu / d + 1u;
}
__device__ __forceinline__ uint32_t udiv(uint32_t n, uint32_t M) {
  return M == 0u ? n : __umulhi(n, M);
}

// Shared-memory elements between the y rows of an xy item of sg densities:
// at least nx*sg and congruent to sg modulo 16, so that the lanes of a warp,
// which take consecutive (y, density) x lines, meet distinct banks.
__host__ __device__ __forceinline__ int plane_pitch(int nx, int sg) {
  return nx * sg + ((16 - ((nx - 1) * sg) % 16) % 16);
}

// Gives the Dirichlet nodes on one line (two mask words, bit k = point k)
// their values: ln[k*ls] = vals[k*vs].
__device__ __forceinline__ void plane_dirichlet(double* ln, int ls, const double* vals,
                                                int64_t vs, unsigned long long w0,
                                                unsigned long long w1) {
  while (w0) {
    const int k = __ffsll((long long)w0) - 1;
    w0 &= w0 - 1;
    ln[k * ls] = __ldg(vals + k * vs);
  }
  while (w1) {
    const int k = 64 + __ffsll((long long)w1) - 1;
    w1 &= w1 - 1;
    ln[k * ls] = __ldg(vals + k * vs);
  }
}

// Forward elimination of one line in shared memory (n points, ls elements
// apart, density s of S); returns q_{n-1}.  The points move through
// registers in batches of kPlaneLineBatch, the next batch loaded before the
// current one is solved and stored, so that the dependent chain of a point
// is one FMA (a load issued after the store of the point before it would
// otherwise wait for that store: the compiler cannot tell them apart).
constexpr int kPlaneLineBatch = 4;

__device__ __forceinline__ double plane_forward(double* ln, int ls, int n, const double2* tab,
                                                int ts) {
  constexpr int B = kPlaneLineBatch;
  double q = 0.0;
  int k0 = 0;
  // whole batches: the next batch is loaded before this one is solved
  if (n >= B) {
    double cur[B];
#pragma unroll
    for (int i = 0; i < B; ++i) cur[i] = ln[i * ls];
    for (; k0 + B <= n; k0 += B) {
      double nxt[B];
      const bool more = k0 + 2 * B <= n;
#pragma unroll
      for (int i = 0; i < B; ++i) nxt[i] = more ? ln[(k0 + B + i) * ls] : 0.0;
      double2 c[B];
#pragma unroll
      for (int i = 0; i < B; ++i) c[i] = tab[(k0 + i) * ts];  // {1/d_k, a_k}
#pragma unroll
      for (int i = 0; i < B; ++i) {
        q = fma(c[i].y, q, cur[i] * c[i].x);
        ln[(k0 + i) * ls] = q;
      }
#pragma unroll
      for (int i = 0; i < B; ++i) cur[i] = nxt[i];
    }
  }
  for (; k0 < n; ++k0) {
    const double2 c = tab[k0 * ts];
    q = fma(c.y, q, ln[k0 * ls] * c.x);
    ln[k0 * ls] = q;
  }
  return q;
}

// Back substitution of one line whose forward values are in place (x =
// q_{n-1} at the last point), in batches as above.
__device__ __forceinline__ void plane_backward(double* ln, int ls, int n, const double2* tab,
                                               int ts, double x) {
  constexpr int B = kPlaneLineBatch;
  int top = n - 2;  // next point to solve, going down
  if (top + 1 >= B) {
    double cur[B];
#pragma unroll
    for (int i = 0; i < B; ++i) cur[i] = ln[(top - i) * ls];
    for (; top + 1 >= B; top -= B) {
      double nxt[B];
      const bool more = top + 1 >= 2 * B;
#pragma unroll
      for (int i = 0; i < B; ++i) nxt[i] = more ? ln[(top - B - i) * ls] : 0.0;
      double a[B];
#pragma unroll
      for (int i = 0; i < B; ++i) a[i] = tab[(top - i) * ts].y;
#pragma unroll
      for (int i = 0; i < B; ++i) {
        x = fma(a[i], x, cur[i]);
        ln[(top - i) * ls] = x;
      }
#pragma unroll
      for (int i = 0; i < B; ++i) cur[i] = nxt[i];
    }
  }
  for (; top >= 0; --top) {
    x = fma(tab[top * ts].y, x, ln[top * ls]);
    ln[top * ls] = x;
  }
}

// One line solved in place: forward elimination, then back substitution,
// with the line's {1/d_k, a_k} pair of point k at tab[k*ts] (shared memory,
// or the member's table in global memory).  Not inlined: a line's registers
// are allocated apart from the staging loops' (the kernel runs one block of
// 512 threads per SM, 128 registers each).
__device__ __noinline__ void plane_line(double* ln, int ls, int n, const double2* tab, int ts) {
  const double q = plane_forward(ln, ls, n, tab, ts);
  plane_backward(ln, ls, n, tab, ts, q);
}

// Copies the {1/d, a} pairs of points 0..n-1, densities s0..s0+cnt-1, of a
// member's axis table (pairs [point][S], 16-byte aligned) into shared memory
// as [point][cnt], with asynchronous 16-byte copies that bypass L1 (waited
// for with the plane's copies).
__device__ __forceinline__ void plane_stage_pairs(double2* dst, const double* k1, int n, int s0,
                                                  int cnt, int S) {
  const double2* src = reinterpret_cast<const double2*>(k1);
  const uint32_t M = udiv_magic((uint32_t)cnt);
  for (int w = threadIdx.x; w < n * cnt; w += blockDim.x) {
    const int k = (int)udiv((uint32_t)w, M);
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + w);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d),
                 "l"(src + k * S + s0 + (w - k * cnt))
                 : "memory");
  }
}

// Copies between a member's field and shared memory, row by row: row r
// (0 <= r < rows) of rl elements sits at sm + r*spitch in shared memory and
// at g + r*gpitch in global memory, where element u of the row is at u when
// the row is contiguous (ud == 0), else at (u / ud)*S + u % ud (ud densities
// of each voxel's S).  Each warp takes whole rows and its lanes step through
// a row 32 elements apart (the global offset of element u advanced without
// division).  Offsets inside a member fit in 32 bits.
//
// Loads are asynchronous copies (cp.async, 8 bytes each) that a thread
// issues for all its elements before waiting for any, so the whole item is
// in flight at once; the caller's block barrier follows the wait.  The field
// a block reads was written by other SMs before the grid barrier that
// precedes the phase, whose acquire makes those writes visible.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <bool LOAD>
__device__ __noinline__ void plane_copy(double* sm, double* g, int rows, int rl, int spitch,
                                        int gpitch, int ud, int S) {
  constexpr int B = kPlaneLoadBatch;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int q32 = ud > 0 ? 32 / ud : 0, r32 = ud > 0 ? 32 - q32 * ud : 0;
  const int x0 = ud > 0 ? lane / ud : 0, d0 = ud > 0 ? lane - x0 * ud : 0;
  for (int r = warp; r < rows; r += nw) {
    double* sr = sm + r * spitch;
    double* gr = g + r * gpitch;
    if (LOAD) {
      if (ud == 0) {
        for (int u = lane; u < rl; u += 32) cp_async8(sr + u, gr + u);
      } else {
        int x = x0, d = d0;
        for (int u = lane; u < rl; u += 32) {
          cp_async8(sr + u, gr + x * S + d);
          x += q32;
          d += r32;
          if (d >= ud) {
            d -= ud;
            ++x;
          }
        }
      }
    } else {
      int x = x0, d = d0;
      for (int u0 = lane; u0 < rl; u0 += 32 * B) {
        int go[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
          go[j] = ud > 0 ? x * S + d : u0 + 32 * j;
          if (ud > 0) {
            x += q32;
            d += r32;
            if (d >= ud) {
              d -= ud;
              ++x;
            }
          }
        }
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (u0 + 32 * j < rl) __stcg(gr + go[j], sr[u0 + 32 * j]);
      }
    }
  }
  if (LOAD) cp_async_wait_all();
}

// The bulk updates (runs of voxels sharing a rate row) and then the agents'
// updates, in list order, of x line `line` of member m, density s, staged in
// shared memory at ln[x*ls] (BioFVM_microenvironment.cpp:603-609,
// BioFVM_basic_agent.cpp:234-235; the operations of bulk_update and
// cell_update).
__device__ __forceinline__ void plane_line_sources(double* ln, int ls, const StepMember& m,
                                                   int64_t line, int s, double dt) {
  const int S = m.S;
  if (m.bulk) {
    const int r1 = __ldg(m.xrun_off + line + 1);
    for (int r = __ldg(m.xrun_off + line); r < r1; ++r) {
      const int4 run = __ldg(m.xruns + r);  // {first x, end x, entry}
      const double add = __dmul_rn(dt, __ldg(m.est + (int64_t)run.z * S + s));
      const double den = __dadd_rn(__dmul_rn(__ldg(m.esu + (int64_t)run.z * S + s), dt), 1.0);
      for (int x = run.x; x < run.y; ++x) ln[x * ls] = __ddiv_rn(__dadd_rn(ln[x * ls], add), den);
    }
  }
  if (m.cells) {
    const int a1 = __ldg(m.xag_off + line + 1);
    const int64_t v0 = line * m.nx;
    for (int r = __ldg(m.xag_off + line); r < a1; ++r) {
      const int x = (int)((int64_t)__ldg(m.ag_key + r) - v0);
      const int64_t ai = __ldg(m.ag_idx + r);
      ln[x * ls] = cell_update(ln[x * ls], __ldg(m.ag_t1 + ai * S + s), __ldg(m.ag_t2 + ai * S + s));
    }
  }
}

// xy item `it` of member m: plane z = it / groups, densities
// [g*psg, g*psg + sg) with g = it % groups.
__device__ __noinline__ void plane_xy_item(const StepMember& m, int it, double* sm,
                                              bool sources, double dt) {
  const int S = m.S, nx = m.nx, ny = m.ny;
  const int z = it / m.pgroups;
  const int g = it - z * m.pgroups;
  const int s0 = g * m.psg;
  const int sg = min(m.psg, S - s0);
  const int pitch = plane_pitch(nx, sg);
  const int row = nx * sg;
  double* gp = m.p + (int64_t)z * nx * ny * S + s0;
  double2* tx = reinterpret_cast<double2*>(sm + kPlaneSmemDoubles);  // [nx][sg]
  double2* ty = tx + nx * sg;                                           // [ny][sg]
  plane_stage_pairs(tx, m.ck1[0], nx, s0, sg, S);
  plane_stage_pairs(ty, m.ck1[1], ny, s0, sg, S);
  plane_copy<true>(sm, gp, ny, row, pitch, nx * S, sg == S ? 0 : sg, S);
  __syncthreads();
  const bool src = sources && (m.bulk || m.cells);
  const uint32_t Msg = udiv_magic((uint32_t)sg);
  const int nt = blockDim.x;
  // x lines: (y, density)
  for (int l = threadIdx.x; l < ny * sg; l += nt) {
    const int y = (int)udiv((uint32_t)l, Msg);
    const int d = l - y * sg;
    const int s = s0 + d;
    double* ln = sm + y * pitch + d;
    if (src) plane_line_sources(ln, sg, m, (int64_t)z * ny + y, s, dt);
    if (m.dirichlet) {
      const int64_t line = (int64_t)z * ny + y;  // x line k*ny + j
      plane_dirichlet(ln, sg, m.dir_field + line * nx * S + s, S,
                      __ldg(m.dir_mask[0] + 2 * line), __ldg(m.dir_mask[0] + 2 * line + 1));
    }
    plane_line(ln, sg, nx, tx + d, sg);
  }
  __syncthreads();
  // y lines: (x, density), consecutive in a row
  for (int l = threadIdx.x; l < row; l += nt) {
    const int x = (int)udiv((uint32_t)l, Msg);
    const int d = l - x * sg;
    const int s = s0 + d;
    double* ln = sm + l;
    if (m.dirichlet) {
      const int64_t line = (int64_t)z * nx + x;  // y line k*nx + i
      plane_dirichlet(ln, pitch, m.dir_field + ((int64_t)z * ny * nx + x) * S + s,
                      (int64_t)nx * S, __ldg(m.dir_mask[1] + 2 * line),
                      __ldg(m.dir_mask[1] + 2 * line + 1));
    }
    plane_line(ln, pitch, ny, ty + d, sg);
  }
  __syncthreads();
  plane_copy<false>(sm, gp, ny, row, pitch, nx * S, sg == S ? 0 : sg, S);
}

// z item `it` of member m: xz plane y = it / strips, columns
// [c0, c0 + cw) of its nx*S (x, density) columns, c0 = (it % strips) * pcw.
__device__ __noinline__ void plane_z_item(const StepMember& m, int it, double* sm) {
  const int S = m.S, nx = m.nx, ny = m.ny, nz = m.nz;
  const int y = it / m.pstrips;
  const int strip = it - y * m.pstrips;
  const int C = nx * S;
  const int c0 = strip * m.pcw;
  const int cw = min(m.pcw, C - c0);
  const int64_t zs = (int64_t)nx * ny * S;  // elements between z planes
  double* gp = m.p + (int64_t)y * C + c0;
  // the z pairs of every density in shared memory when they fit, else read
  // from the member's table
  const bool staged = nz * S <= kPlaneTabPairs;
  double2* tz = reinterpret_cast<double2*>(sm + kPlaneSmemDoubles);  // [nz][S]
  if (staged) plane_stage_pairs(tz, m.ck1[2], nz, 0, S, S);
  const double2* tzs = staged ? tz : reinterpret_cast<const double2*>(m.ck1[2]);
  plane_copy<true>(sm, gp, nz, cw, cw, (int)zs, 0, S);
  __syncthreads();
  const uint32_t MS = udiv_magic((uint32_t)S);
  for (int l = threadIdx.x; l < cw; l += blockDim.x) {
    const int col = c0 + l;
    const int x = (int)udiv((uint32_t)col, MS);
    const int s = col - x * S;
    double* ln = sm + l;
    const int64_t zline = (int64_t)y * nx + x;  // z line j*nx + i
    if (m.dirichlet)
      plane_dirichlet(ln, cw, m.dir_field + zline * S + s, zs, __ldg(m.dir_mask[2] + 2 * zline),
                      __ldg(m.dir_mask[2] + 2 * zline + 1));
    plane_line(ln, cw, nz, tzs + s, S);
  }
  __syncthreads();
  plane_copy<false>(sm, gp, nz, cw, cw, (int)zs, 0, S);
}

// Runs the items of one phase: item indices come from *ctr (one atomicAdd
// per item, issued one item ahead by thread 0); members are numbered in
// order, so a block's member index only advances.
template <int PH>
__device__ __forceinline__ void plane_phase(const BatchStepsArgs& a, int* ctr, double* sm,
                                            int* s_item) {
  const int64_t nitems = a.tiles[PH];
  if (threadIdx.x == 0) *s_item = atomicAdd(ctr, 1);
  __syncthreads();
  int cur = *s_item;
  int mi = 0;
  while (cur < nitems) {
    int nxt = 0;
    if (threadIdx.x == 0) nxt = atomicAdd(ctr, 1);
    while (mi + 1 < a.nmem && __ldg(&a.mem[mi + 1].tile0[PH]) <= cur) ++mi;
    const StepMember& m = a.mem[mi];
    if (PH == 0)
      plane_xy_item(m, (int)(cur - m.tile0[0]), sm, a.sources != 0, a.dt);
    else
      plane_z_item(m, (int)(cur - m.tile0[2]), sm);
    __syncthreads();  // shared memory and *s_item are free again
    if (threadIdx.x == 0) *s_item = nxt;
    __syncthreads();
    cur = *s_item;
  }
}

// nsteps whole steps of every member in the plane form; launched
// cooperatively with kPlaneThreads threads and kPlaneSmemDoubles doubles +
// kPlaneTabPairs pairs of dynamic shared memory per block.  a.tiles[0] / a.tiles[2] are the xy / z
// items of a phase; a.ctr holds 2 * nsteps zeroed counters; a.sources: the
// members' bulk and cell updates run (their runs and agent offsets are in
// place).
__global__ void __launch_bounds__(kPlaneThreads, 1) batch_planes_kernel(const BatchStepsArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) double plane_smem[];
  __shared__ int s_item;
  for (int step = 0; step < a.nsteps; ++step) {
    plane_phase<0>(a, a.ctr + 2 * step, plane_smem, &s_item);
    grid.sync();
    plane_phase<2>(a, a.ctr + 2 * step + 1, plane_smem, &s_item);
    grid.sync();
  }
}

// Per x line of member m (line = k*ny + j, 0..ny*nz), the first sorted
// agent at or past the line's first voxel (the agents' voxel keys ascend).
static __global__ void plane_agent_lines_kernel(StepMember m, int* __restrict__ xag_off) {
  const int64_t lines = (int64_t)m.ny * m.nz;
  const int64_t line = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (line > lines) return;
  const uint64_t v = (uint64_t)(line * m.nx);
  int64_t lo = 0, hi = m.nagents;
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (m.ag_key[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  xag_off[line] = (int)lo;
}

}  // namespace bfvm
