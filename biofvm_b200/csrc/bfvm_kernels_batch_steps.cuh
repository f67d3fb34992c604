// Whole steps of a group of independent microenvironments in one persistent
// cooperative launch (the persistent mode of bfvm_batch).
//
// A group is a set of FP64 instances whose fields together fit in L2 and whose
// lines are at most 128 points.  One launch over all SMs runs all n steps of
// every member: the phases of a step are shared by the members and separated
// by grid-wide barriers of the cooperative launch (every block is resident,
// so each barrier completes), and the fields stay in L2 from phase to phase
// and from step to step.  Per step, for every member (its own mesh, densities,
// Thomas tables and lists; BioFVM_solvers.cpp:77-276 on one Microenvironment
// each):
//   sources (first step of a call only): per bulk entry its update
//            (BioFVM_microenvironment.cpp:603-609), then its voxel's agents in
//            list order (BioFVM_basic_agent.cpp:234-235); per agent voxel
//            without a bulk entry its agents;
//   x, y, z: work items are (member, tile) pairs, a tile being TW lines x NC
//            chunks of CH points of one member (TW = 128 / NC), solved as the
//            register sweep kernel solves them (chunk-local passes, the chunks'
//            carries folded through shared memory, fix-ups); as a chunk is
//            loaded, its Dirichlet nodes take their values (before each axis,
//            BioFVM_solvers.cpp:177, 207, 241; 128-bit masks per line mark
//            them); as the z phase stores a point, the next step's bulk and
//            cell updates of that voxel are applied (each voxel lies on exactly
//            one z chunk, so its thread is the only one to touch it before the
//            next x phase), which saves the sources phase of later steps.
// Work items of a phase are numbered member after member; a block takes items
// blockIdx.x, blockIdx.x + gridDim.x, ..., so its member index only advances.
#pragma once

#include <cooperative_groups.h>

#include "bfvm_kernels.cuh"
#include "bfvm_kernels_tma.cuh"

namespace bfvm {

constexpr int kBatchStepsMaxN = 128;  // points per axis of a member (two mask words)
constexpr int kBatchStepsThreads = 128;
constexpr int kBatchLineBatch = 4;  // line form: points per load batch

// One member of a group (device copy; read through the read-only cache).
struct StepMember {
  double* p;  // [nz][ny][nx][S]
  int nx, ny, nz, S;
  int nc[3], tw[3];    // per axis: chunks per line, columns per tile
  int64_t ncols[3];    // per axis: (line, density) columns
  int64_t tile0[3];    // per axis: first work item of this member in the phase
  int64_t src0, nsrc;  // sources work items of the first step: [src0, src0 + nsrc)
  AxisCoef<double> coef[3];
  int bulk, cells, dirichlet;
  // voxel maps: bulk rate row (or -1) and first sorted agent (or -1)
  const int* bulk_map;
  const int* ag_map;
  // per z line (j*nx + i): bit k set when voxel (i, j, k) has a bulk entry or
  // agents (two words); the maps are read only there
  const unsigned long long* src_mask;
  // bulk rates of row r, density s: S*T at st[(r*S + s)*rs], U+S at su[...]
  const double* st;
  const double* su;
  int rs;
  int64_t nbulk;
  const int64_t* bulk_vox;  // [E] ascending (first step's sources)
  const int* bulk_row;      // row of entry e (nullptr: row = e)
  int64_t nagents;
  const uint64_t* ag_key;  // sorted voxel keys (stable in list order)
  const int* ag_idx;       // list position of each sorted entry
  const double* ag_t1;     // [A][S] in list order
  const double* ag_t2;
  // Dirichlet nodes: per axis and line two mask words, and the node values
  // at their places in a field-shaped array [N][S]
  const unsigned long long* dir_mask[3];
  const double* dir_field;
  // tile form: per axis the chunk tables of 32-point chunks, chunk c at
  // k1 + c*32*S*2 and kg alike ({1/d, a} and {G, R} per point and density),
  // kc [nc][S][4] the per-chunk transfer constants
  const double* ck1[3];
  const double* ckg[3];
  const double* ckc[3];
  // plane form: densities per xy item (psg) and items per xy plane
  // (pgroups); columns per z item (pcw) and items per xz plane (pstrips);
  // tile0[0] / tile0[2] are the member's first xy / z items
  int psg, pgroups, pcw, pstrips;
  // plane form, sources by x line (line = k*ny + j): bulk runs {first x, end
  // x, entry} of line at xruns[xrun_off[line] .. xrun_off[line+1]), rates of
  // entry e at est / esu [e*S + s]; sorted agents of the line from
  // xag_off[line] to xag_off[line+1]
  const int* xrun_off;
  const int4* xruns;
  const double* est;
  const double* esu;
  const int* xag_off;
};

struct BatchStepsArgs {
  const StepMember* mem;
  int nmem;
  int64_t tiles[3];  // work items of each axis phase
  int64_t src_items;
  int nsteps;
  double dt;
  int sources;  // any member has bulk or cell updates to apply
  int* ctr;     // plane form: 2 * nsteps work-item counters, zeroed before the launch
};

__device__ __forceinline__ double member_cells(const StepMember& m, double x, int r, uint64_t vox,
                                               int s) {
  do {
    const int64_t ai = __ldg(m.ag_idx + r);
    x = cell_update(x, __ldg(m.ag_t1 + ai * m.S + s), __ldg(m.ag_t2 + ai * m.S + s));
    ++r;
  } while (r < m.nagents && __ldg(m.ag_key + r) == vox);
  return x;
}

__device__ __forceinline__ double member_bulk(const StepMember& m, double x, int row, int s,
                                              double dt) {
  const int64_t q = ((int64_t)row * m.S + s) * m.rs;
  return bulk_update(x, __ldg(m.st + q), __ldg(m.su + q), dt);
}

// Sources work item w (< nsrc) of member m: bulk entries first (each with its
// voxel's agents), then the agent voxels without a bulk entry.
__device__ __forceinline__ void member_sources(const StepMember& m, int64_t w, double dt) {
  const int S = m.S;
  const int64_t nb = m.bulk ? m.nbulk * S : 0;
  if (w < nb) {
    const int64_t e = w / S;
    const int s = (int)(w - e * S);
    const int64_t vox = __ldg(m.bulk_vox + e);
    double* q = m.p + vox * S + s;
    const int row = m.bulk_row ? __ldg(m.bulk_row + e) : (int)e;
    double x = member_bulk(m, *q, row, s, dt);
    if (m.cells) {
      const int r = __ldg(m.ag_map + vox);
      if (r >= 0) x = member_cells(m, x, r, (uint64_t)vox, s);
    }
    *q = x;
  } else {
    const int64_t r = (w - nb) / S;
    const int s = (int)(w - nb - r * S);
    const uint64_t vox = __ldg(m.ag_key + r);
    if (r > 0 && __ldg(m.ag_key + r - 1) == vox) return;  // not the voxel's first agent
    if (m.bulk && __ldg(m.bulk_map + vox) >= 0) return;   // done with its bulk entry
    double* q = m.p + (int64_t)vox * S + s;
    *q = member_cells(m, *q, (int)r, vox, s);
  }
}

// Two mask words of a line -> the bits of the chunk starting at k0 (the chunk
// length divides 64, so a chunk never straddles the words).
__device__ __forceinline__ unsigned long long chunk_bits(const unsigned long long* mask,
                                                         int64_t line, int k0) {
  return __ldg(mask + 2 * line + (k0 >> 6)) >> (k0 & 63);
}

// One tile of member m along axis AX.  sm holds 4 * 128 carries.
template <int AX, int CH>
__device__ __forceinline__ void member_tile(const StepMember& m, int64_t tile, double* sm,
                                            bool sources_after, double dt) {
  const int S = m.S;
  const int64_t plane = (int64_t)m.nx * m.ny;
  const int n = AX == 0 ? m.nx : (AX == 1 ? m.ny : m.nz);
  const int64_t C = AX == 0 ? S : (AX == 1 ? (int64_t)m.nx * S : plane * S);
  const int64_t outer_stride = AX == 0 ? (int64_t)m.nx * S : (AX == 1 ? plane * S : 0);
  const int64_t ls = C;  // elements between consecutive points of a line
  const int64_t ncols = m.ncols[AX];
  const int NC = m.nc[AX];
  const int TW = m.tw[AX];
  const int tx = threadIdx.x % TW;
  const int c = threadIdx.x / TW;  // chunk; threads past NC chunks idle
  const bool in_tile = c < NC;
  const int k0 = c * CH;
  double* sQ = sm;  // [NC][TW] forward chunk end values
  double* sP = sQ + NC * TW;
  double* sX = sP + NC * TW;  // backward chunk start values
  double* sR = sX + NC * TW;
  const AxisCoef<double> cf = m.coef[AX];
  const int64_t vcol = tile * TW + tx;
  const bool active = in_tile && vcol < ncols;
  const int len = active ? max(0, min(CH, n - k0)) : 0;
  double* ptr = m.p;
  const double* dptr = m.dir_field;
  int s = 0;
  unsigned long long nodes = 0ull;
  if (active) {
    const int64_t outer = vcol / C;
    const int64_t col = vcol - outer * C;
    const int64_t off = outer * outer_stride + col + (int64_t)k0 * ls;
    ptr = m.p + off;
    dptr = m.dir_field + off;
    s = (int)(col % S);
    if (m.dirichlet) nodes = chunk_bits(m.dir_mask[AX], vcol / S, k0);
  }
  // the field moves through L2 only, so that L1 keeps the coefficient tables
  double v[CH];
#pragma unroll
  for (int q = 0; q < CH; ++q)
    v[q] = (q < len) ? (((nodes >> q) & 1ull) ? __ldcg(dptr + q * ls) : __ldcg(ptr + q * ls))
                     : 0.0;
  const double* c_inv = cf.inv_den + (int64_t)k0 * S + s;
  const double* c_fwd = cf.fwd + (int64_t)k0 * S + s;
  const double* c_bwd = cf.bwd + (int64_t)k0 * S + s;
  // forward elimination, chunk-local with carry-in 0
  const double c1 = active ? __ldg(cf.c1 + s) : 0.0;
  double q = 0.0, P = 1.0;
#pragma unroll
  for (int i = 0; i < CH; ++i) {
    if (i < len) {
      q = (v[i] + c1 * q) * __ldg(c_inv + i * S);
      P = P * __ldg(c_fwd + i * S);
      v[i] = q;
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
    for (int i = 0; i < CH; ++i) {
      if (i < len) {
        Pm = Pm * __ldg(c_fwd + i * S);
        v[i] = v[i] + Pm * carry;
      }
    }
  }
  // back substitution, chunk-local with carry-in 0
  double x = 0.0, R = 1.0;
#pragma unroll
  for (int i = CH - 1; i >= 0; --i) {
    if (i < len) {
      const double b = __ldg(c_bwd + i * S);
      x = v[i] + b * x;
      R = R * b;
      v[i] = x;
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
    for (int i = CH - 1; i >= 0; --i) {
      if (i < len) {
        Rm = Rm * __ldg(c_bwd + i * S);
        v[i] = v[i] + Rm * carry;
      }
    }
  }
  if (AX == 2 && sources_after && (m.bulk || m.cells) && len > 0) {
    const int64_t zline = vcol / S;  // j*nx + i
    const unsigned long long flagged = chunk_bits(m.src_mask, zline, k0);
    const int64_t vox0 = zline + (int64_t)k0 * plane;  // voxel of the chunk's point 0
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      if (i < len && ((flagged >> i) & 1ull)) {
        const int64_t vox = vox0 + i * plane;
        double xv = v[i];
        if (m.bulk) {
          const int row = __ldg(m.bulk_map + vox);
          if (row >= 0) xv = member_bulk(m, xv, row, s, dt);
        }
        if (m.cells) {
          const int r = __ldg(m.ag_map + vox);
          if (r >= 0) xv = member_cells(m, xv, r, (uint64_t)vox, s);
        }
        v[i] = xv;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < CH; ++i)
    if (i < len) __stcg(ptr + i * ls, v[i]);
  __syncthreads();  // the carries of this tile are read before the next overwrites them
}

template <int AX, int CH>
__device__ __forceinline__ void batch_axis(const BatchStepsArgs& a, double* sm,
                                           bool sources_after) {
  int mi = 0;
  for (int64_t t = blockIdx.x; t < a.tiles[AX]; t += gridDim.x) {
    while (mi + 1 < a.nmem && __ldg(&a.mem[mi + 1].tile0[AX]) <= t) ++mi;
    const StepMember& m = a.mem[mi];
    member_tile<AX, CH>(m, t - m.tile0[AX], sm, sources_after, a.dt);
  }
}

__device__ __forceinline__ void batch_sources(const BatchStepsArgs& a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int mi = 0;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < a.src_items;
       w += stride) {
    while (mi + 1 < a.nmem && __ldg(&a.mem[mi + 1].src0) <= w) ++mi;
    const StepMember& m = a.mem[mi];
    member_sources(m, w - m.src0, a.dt);
  }
}

// nsteps whole steps of every member, CH-point chunks (8 or 16: lines of up
// to 128 points in at most 16 or 8 chunks); launched cooperatively with 128
// threads and 4 * 128 doubles of dynamic shared memory per block.
template <int CH>
__global__ void __launch_bounds__(kBatchStepsThreads, 6) batch_steps_kernel(const BatchStepsArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double batch_carries[];
  for (int step = 0; step < a.nsteps; ++step) {
    if (a.sources && step == 0) {
      batch_sources(a);
      grid.sync();
    }
    batch_axis<0, CH>(a, batch_carries, false);
    grid.sync();
    batch_axis<1, CH>(a, batch_carries, false);
    grid.sync();
    batch_axis<2, CH>(a, batch_carries, a.sources && step + 1 < a.nsteps);
    grid.sync();
  }
}

// ---- line form: one thread per (line, density) column ---------------------
//
// The same phases with another work split: a work item is one column of one
// member, solved whole by one thread (forward elimination, storing the
// forward values, then back substitution reading them back), so there is no
// fold between chunks and blocks need no barrier; the field crosses L2 twice
// per phase (32 B/VS instead of 16).  Values move in batches of LB points:
// the next batch is loaded before the current one is solved and stored, so
// a thread keeps LB loads in flight.

// Bulk and cell updates of the next step at one stored z-line point.
__device__ __noinline__ double member_point_sources(const StepMember& m, double x,
                                                       int64_t vox, int s, double dt) {
  if (m.bulk) {
    const int row = __ldg(m.bulk_map + vox);
    if (row >= 0) x = member_bulk(m, x, row, s, dt);
  }
  if (m.cells) {
    const int r = __ldg(m.ag_map + vox);
    if (r >= 0) x = member_cells(m, x, r, (uint64_t)vox, s);
  }
  return x;
}

// Loads of one line: points k0 .. k0+LB-1 (those below n), the Dirichlet
// nodes' values where a mask bit is set (DIR).
template <int LB, bool DIR>
__device__ __forceinline__ void line_load(double (&v)[LB], const double* p, const double* d,
                                          int ls, int k0, int n, unsigned long long nd0,
                                          unsigned long long nd1) {
#pragma unroll
  for (int i = 0; i < LB; ++i) {
    const int k = k0 + i;
    if (k < n) {
      bool node = false;
      if (DIR) node = ((k < 64 ? (nd0 >> k) : (nd1 >> (k - 64))) & 1ull) != 0;
      v[i] = node ? __ldcg(d + k * ls) : __ldcg(p + k * ls);
    }
  }
}

// One (line, density) column of member m along axis AX, solved whole: the
// forward values are stored over the field, then read back by the back
// substitution.  Offsets inside a member fit in 32 bits (at most 128^3
// voxels x the densities of an FP64 field that fits L2).  DIR: the line has
// Dirichlet nodes; SRC: the z line has voxels with bulk or agent updates.
template <int AX, int LB, bool DIR, bool SRC>
__device__ __noinline__ void line_solve(const StepMember& m, double* ptr, const double* dptr,
                                           int ls, int n, int s, int line,
                                           unsigned long long nd0, unsigned long long nd1,
                                           unsigned long long sf0, unsigned long long sf1,
                                           double dt) {
  const int S = m.S;
  const AxisCoef<double> cf = m.coef[AX];
  const double c1 = __ldg(cf.c1 + s);
  const double* inv = cf.inv_den + s;
  const double* bwd = cf.bwd + s;
  double cur[LB], nxt[LB];
  line_load<LB, DIR>(cur, ptr, dptr, ls, 0, n, nd0, nd1);
  double q = 0.0;
  for (int k0 = 0; k0 < n; k0 += LB) {
    line_load<LB, DIR>(nxt, ptr, dptr, ls, k0 + LB, n, nd0, nd1);
#pragma unroll
    for (int i = 0; i < LB; ++i) {
      const int k = k0 + i;
      if (k < n) {
        q = (cur[i] + c1 * q) * __ldg(inv + k * S);
        __stcg(ptr + k * ls, q);
      }
    }
#pragma unroll
    for (int i = 0; i < LB; ++i) cur[i] = nxt[i];
  }
  // back substitution from the last point (x = q there)
  const int plane = m.nx * m.ny;
  double x = q;
  if (SRC && (((n - 1) < 64 ? (sf0 >> (n - 1)) : (sf1 >> (n - 65))) & 1ull))
    ptr[(n - 1) * ls] = member_point_sources(m, x, (int64_t)line + (int64_t)(n - 1) * plane, s, dt);
#pragma unroll
  for (int i = 0; i < LB; ++i)
    if (n - 2 - i >= 0) cur[i] = __ldcg(ptr + (n - 2 - i) * ls);
  for (int top = n - 2; top >= 0; top -= LB) {
#pragma unroll
    for (int i = 0; i < LB; ++i)
      if (top - LB - i >= 0) nxt[i] = __ldcg(ptr + (top - LB - i) * ls);
#pragma unroll
    for (int i = 0; i < LB; ++i) {
      const int k = top - i;
      if (k >= 0) {
        x = cur[i] + __ldg(bwd + k * S) * x;
        double out = x;
        if (SRC && ((k < 64 ? (sf0 >> k) : (sf1 >> (k - 64))) & 1ull))
          out = member_point_sources(m, x, (int64_t)line + (int64_t)k * plane, s, dt);
        __stcg(ptr + k * ls, out);
      }
    }
#pragma unroll
    for (int i = 0; i < LB; ++i) cur[i] = nxt[i];
  }
}

template <int AX, int LB>
__device__ __forceinline__ void member_line(const StepMember& m, int vcol, bool sources_after,
                                            double dt) {
  const int S = m.S;
  const int plane = m.nx * m.ny;
  const int n = AX == 0 ? m.nx : (AX == 1 ? m.ny : m.nz);
  const int C = AX == 0 ? S : (AX == 1 ? m.nx * S : plane * S);
  const int outer_stride = AX == 0 ? m.nx * S : (AX == 1 ? plane * S : 0);
  const int outer = vcol / C;
  const int col = vcol - outer * C;
  const int s = col % S;
  const int off = outer * outer_stride + col;
  const int line = vcol / S;  // x: k*ny + j; y: k*nx + i; z: j*nx + i
  double* ptr = m.p + off;
  const double* dptr = m.dir_field + off;
  unsigned long long nd0 = 0ull, nd1 = 0ull;
  if (m.dirichlet) {
    nd0 = __ldg(m.dir_mask[AX] + 2 * line);
    nd1 = __ldg(m.dir_mask[AX] + 2 * line + 1);
  }
  unsigned long long sf0 = 0ull, sf1 = 0ull;
  if (AX == 2 && sources_after && (m.bulk || m.cells)) {
    sf0 = __ldg(m.src_mask + 2 * line);
    sf1 = __ldg(m.src_mask + 2 * line + 1);
  }
  const bool dir = (nd0 | nd1) != 0ull, src = (sf0 | sf1) != 0ull;
  if (dir) {
    if (src)
      line_solve<AX, LB, true, true>(m, ptr, dptr, C, n, s, line, nd0, nd1, sf0, sf1, dt);
    else
      line_solve<AX, LB, true, false>(m, ptr, dptr, C, n, s, line, nd0, nd1, sf0, sf1, dt);
  } else {
    if (src)
      line_solve<AX, LB, false, true>(m, ptr, dptr, C, n, s, line, nd0, nd1, sf0, sf1, dt);
    else
      line_solve<AX, LB, false, false>(m, ptr, dptr, C, n, s, line, nd0, nd1, sf0, sf1, dt);
  }
}

template <int AX, int LB>
__device__ __forceinline__ void batch_axis_lines(const BatchStepsArgs& a, bool sources_after) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int mi = 0;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < a.tiles[AX];
       w += stride) {
    while (mi + 1 < a.nmem && __ldg(&a.mem[mi + 1].tile0[AX]) <= w) ++mi;
    const StepMember& m = a.mem[mi];
    member_line<AX, LB>(m, (int)(w - m.tile0[AX]), sources_after, a.dt);
  }
}

// nsteps whole steps of every member in the line form (work items: columns,
// tile0 = first column of a member in each phase); launched cooperatively
// with kBatchStepsThreads threads and no shared memory.
template <int LB>
__global__ void __launch_bounds__(kBatchStepsThreads, 8) batch_lines_kernel(const BatchStepsArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  for (int step = 0; step < a.nsteps; ++step) {
    if (a.sources && step == 0) {
      batch_sources(a);
      grid.sync();
    }
    batch_axis_lines<0, LB>(a, false);
    grid.sync();
    batch_axis_lines<1, LB>(a, false);
    grid.sync();
    batch_axis_lines<2, LB>(a, a.sources && step + 1 < a.nsteps);
    grid.sync();
  }
}

// ---- tile form: 32-point chunks with the sweep kernels' chunk tables -------
//
// A work item is a tile of 32 columns x NC <= 4 chunks of 32 points of one
// member (128 threads), loaded straight from global memory (32 loads in
// flight per thread) and solved with the chunk tables of the TMA sweep
// kernels (chunk_local / chunk_carries / chunk_fix: three table loads per
// point, the fold over at most four chunks).

constexpr int kBatchTileCols = 32;
constexpr int kBatchTileCh = 32;

// Chunk tables of member m for axis AX in shared memory: k1 | kg | kc, each
// section 16-byte aligned (the layout of the member's own table buffer).
// Returns the number of doubles.
template <int AX>
__device__ __forceinline__ int tile_tables_doubles(const StepMember& m) {
  const int n = AX == 0 ? m.nx : (AX == 1 ? m.ny : m.nz);
  const int nc = (n + kBatchTileCh - 1) / kBatchTileCh;
  const int kx = nc * kBatchTileCh * m.S * 2;
  return 2 * kx + nc * m.S * 4;
}

template <int AX>
__device__ __forceinline__ void stage_tile_tables(const StepMember& m, double* tab) {
  // k1 and kg are adjacent in the member's buffer (kx doubles each, kx even)
  // and kc follows kg directly: one contiguous copy
  const int nd = tile_tables_doubles<AX>(m);
  const double2* src = reinterpret_cast<const double2*>(m.ck1[AX]);
  double2* dst = reinterpret_cast<double2*>(tab);
  for (int i = threadIdx.x; i < nd / 2; i += blockDim.x) dst[i] = __ldcg(src + i);
}

template <int AX>
__device__ __forceinline__ void member_tile32(const StepMember& m, int tile, Pair<double>* fold,
                                              const double* tab, bool sources_after, double dt) {
  constexpr int CH = kBatchTileCh, W = kBatchTileCols;
  const int S = m.S;
  const int plane = m.nx * m.ny;
  const int n = AX == 0 ? m.nx : (AX == 1 ? m.ny : m.nz);
  const int C = AX == 0 ? S : (AX == 1 ? m.nx * S : plane * S);
  const int outer_stride = AX == 0 ? m.nx * S : (AX == 1 ? plane * S : 0);
  const int ls = C;
  const int NC = m.nc[AX];
  const int kx = NC * CH * S * 2;
  const double* k1 = tab;
  const double* kg = tab + kx;
  const int tx = threadIdx.x % W;
  const int c = threadIdx.x / W;  // chunk; threads past NC chunks idle
  const int k0 = c * CH;
  const int vcol = tile * W + tx;
  const bool active = c < NC && vcol < (int)m.ncols[AX];
  const int len = active ? max(0, min(CH, n - k0)) : 0;
  int s = 0, line = 0;
  double* ptr = m.p;
  const double* dptr = m.dir_field;
  unsigned long long nodes = 0ull;
  if (active) {
    const int outer = vcol / C;
    const int col = vcol - outer * C;
    s = col % S;
    line = vcol / S;
    const int off = outer * outer_stride + col + k0 * ls;
    ptr += off;
    dptr += off;
    if (m.dirichlet) nodes = chunk_bits(m.dir_mask[AX], line, k0);
  }
  // the field moves through L2 only (__ldcg / __stcg); the tables are in
  // shared memory
  double v[CH];
  if (nodes == 0ull) {
#pragma unroll
    for (int i = 0; i < CH; ++i) v[i] = (i < len) ? __ldcg(ptr + i * ls) : 0.0;
  } else {
#pragma unroll
    for (int i = 0; i < CH; ++i)
      v[i] = (i < len) ? (((nodes >> i) & 1ull) ? __ldcg(dptr + i * ls) : __ldcg(ptr + i * ls))
                       : 0.0;
  }
  const int row = (k0 * S + s) * 2;
  double qe = 0.0, x0 = 0.0;
  chunk_local<true, double, CH>(v, len, k1 + row, S, qe, x0);
  if (c < NC) st_fold(fold + c * W + tx, qe, x0);
  __syncthreads();
  if (len > 0) {
    ChunkCoef<double> ct;
    ct.kc = tab + 2 * kx;
    double cf, cb;
    chunk_carries<true, double>(fold, W, tx, c, NC, ct, s, S, cf, cb);
    chunk_fix<true, double, CH>(v, len, kg + row, S, cf, cb);
    if (AX == 2 && sources_after && (m.bulk || m.cells)) {
      const unsigned long long flagged = chunk_bits(m.src_mask, line, k0);
      if (flagged != 0ull) {
        const int64_t vox0 = (int64_t)line + (int64_t)k0 * plane;
#pragma unroll
        for (int i = 0; i < CH; ++i)
          if (i < len && ((flagged >> i) & 1ull))
            v[i] = member_point_sources(m, v[i], vox0 + (int64_t)i * plane, s, dt);
      }
    }
#pragma unroll
    for (int i = 0; i < CH; ++i)
      if (i < len) __stcg(ptr + i * ls, v[i]);
  }
  __syncthreads();  // the fold of this tile is read before the next overwrites it
}

template <int AX>
__device__ __forceinline__ void batch_axis_tiles(const BatchStepsArgs& a, Pair<double>* fold,
                                                 double* tab, bool sources_after) {
  int mi = 0, staged = -1;
  for (int64_t t = blockIdx.x; t < a.tiles[AX]; t += gridDim.x) {
    while (mi + 1 < a.nmem && __ldg(&a.mem[mi + 1].tile0[AX]) <= t) ++mi;
    const StepMember& m = a.mem[mi];
    if (mi != staged) {  // this member's tables for this axis into shared memory
      stage_tile_tables<AX>(m, tab);
      __syncthreads();
      staged = mi;
    }
    member_tile32<AX>(m, (int)(t - m.tile0[AX]), fold, tab, sources_after, a.dt);
  }
  __syncthreads();  // the tables are restaged by the next phase
}

// nsteps whole steps of every member in the tile form; launched
// cooperatively with 128 threads and, in dynamic shared memory, 4 x 32
// (qe, x0) pairs plus the largest member's chunk tables of one axis.
__global__ void __launch_bounds__(kBatchStepsThreads, 2) batch_tiles_kernel(const BatchStepsArgs a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char tiles_smem[];
  Pair<double>* fold = reinterpret_cast<Pair<double>*>(tiles_smem);
  double* tab = reinterpret_cast<double*>(fold + 4 * kBatchTileCols);
  for (int step = 0; step < a.nsteps; ++step) {
    if (a.sources && step == 0) {
      batch_sources(a);
      grid.sync();
    }
    batch_axis_tiles<0>(a, fold, tab, false);
    grid.sync();
    batch_axis_tiles<1>(a, fold, tab, false);
    grid.sync();
    batch_axis_tiles<2>(a, fold, tab, a.sources && step + 1 < a.nsteps);
    grid.sync();
  }
}

// A member's maps (bulk_map and ag_map -1, masks 0 beforehand): bulk rate row
// and first sorted agent per voxel, the z-line source masks, the Dirichlet
// nodes' line masks (two words per line) and values at their places.
static __global__ void batch_maps_kernel(StepMember m, const int64_t* __restrict__ dir_vox,
                                         const double* __restrict__ dir_val, int64_t ndir,
                                         int* __restrict__ bulk_map, int* __restrict__ ag_map,
                                         unsigned long long* __restrict__ src_mask,
                                         unsigned long long* __restrict__ mx,
                                         unsigned long long* __restrict__ my,
                                         unsigned long long* __restrict__ mz,
                                         double* __restrict__ dir_field) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t plane = (int64_t)m.nx * m.ny;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
       i < m.nbulk || i < m.nagents || i < ndir; i += stride) {
    if (i < m.nbulk) {
      const int64_t v = m.bulk_vox[i];
      bulk_map[v] = m.bulk_row ? m.bulk_row[i] : (int)i;
      const int64_t k = v / plane;
      atomicOr(src_mask + 2 * (v - k * plane) + (k >> 6), 1ull << (k & 63));
    }
    if (i < m.nagents && (i == 0 || m.ag_key[i] != m.ag_key[i - 1])) {
      const int64_t v = (int64_t)m.ag_key[i];
      ag_map[v] = (int)i;
      const int64_t k = v / plane;
      atomicOr(src_mask + 2 * (v - k * plane) + (k >> 6), 1ull << (k & 63));
    }
    if (i < ndir) {
      const int64_t v = dir_vox[i];
      const int64_t k = v / plane, ij = v - k * plane, j = ij / m.nx, ii = ij - j * m.nx;
      atomicOr(mx + 2 * (v / m.nx) + (ii >> 6), 1ull << (ii & 63));
      atomicOr(my + 2 * (k * m.nx + ii) + (j >> 6), 1ull << (j & 63));
      atomicOr(mz + 2 * ij + (k >> 6), 1ull << (k & 63));
      for (int s = 0; s < m.S; ++s) dir_field[v * m.S + s] = dir_val[i * m.S + s];
    }
  }
}

}  // namespace bfvm
