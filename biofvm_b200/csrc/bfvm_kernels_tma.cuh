// Persistent, TMA-fed LOD sweep kernels (sm_100a).
//
// The Thomas solve of one line (BioFVM_solvers.cpp:186-200) is cut into
// chunks of CH points, one chunk per thread, held in registers.  With the
// per-chunk tables of chunk_tables() (bfvm_host_math.h) a chunk is solved as
//   forward   q'_k = a_k q'_{k-1} + p_k / d_k        (carry-in 0)
//   backward  x'_k = a_k x'_{k+1} + q'_k   (a_k = c1/d_k = -cx_k; carry-in 0)
//   fix-up    x_k  = x'_k + cf * G_k + cb * R_k
// where cf / cb are the true forward / backward carries into the chunk.  They
// come from one pass over the chunks of the line (one shared-memory fold, a
// single barrier per tile).  Every density element is read once and written
// once per sweep; the per-point work is one multiply and four FMAs, and the
// tables are interleaved [point][density] so that a warp's coefficient loads
// are contiguous.
//
//  lod_lines_tma_kernel  (y and z sweeps) -- a tile is W consecutive columns
//    (contiguous in memory) x all n points of their lines, fetched with a 3-D
//    tensor map as a [n][W] box into a ring of shared-memory stages; the stage
//    is refilled as soon as the tile is in registers, and results go from
//    registers to global memory with coalesced stores.
//
//  lod_rows_tma_kernel  (x sweep) -- a tile is R whole rows (R*nx*S
//    contiguous elements), fetched with one 1-D bulk copy.  The rest of the
//    step is applied to each thread's chunk in registers before the sweep
//    (bulk sources/sinks, cell sources/sinks in agent-list order, the
//    Dirichlet overwrite) and the Dirichlet overwrite again after it; then
//    the rows go back to shared memory and one 1-D bulk store writes them.
//
// Waits are bounded (bfvm_tma.cuh); on a timeout the block records status 1,
// waits (bounded) for its copies still in flight, and returns.
#pragma once

#include "bfvm_kernels.cuh"
#include "bfvm_tma.cuh"

#include <type_traits>

namespace bfvm {

template <typename T>
struct __align__(2 * sizeof(T)) Pair {
  T x, y;
};
// SMEM: the tables were staged in shared memory (plain loads), else global
// read-only loads.
template <bool SMEM>
__device__ __forceinline__ Pair<double> ld_pair(const double* p) {
  const double2 v = SMEM ? *reinterpret_cast<const double2*>(p)
                         : __ldg(reinterpret_cast<const double2*>(p));
  return {v.x, v.y};
}
template <bool SMEM>
__device__ __forceinline__ Pair<float> ld_pair(const float* p) {
  const float2 v = SMEM ? *reinterpret_cast<const float2*>(p)
                        : __ldg(reinterpret_cast<const float2*>(p));
  return {v.x, v.y};
}
template <bool SMEM, typename T>
__device__ __forceinline__ T ld_one(const T* p) {
  return SMEM ? *p : __ldg(p);
}
// (qe, x0) pairs of the fold in shared memory, read and written as one vector
__device__ __forceinline__ Pair<double> ld_fold(const Pair<double>* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  return {v.x, v.y};
}
__device__ __forceinline__ Pair<float> ld_fold(const Pair<float>* p) {
  const float2 v = *reinterpret_cast<const float2*>(p);
  return {v.x, v.y};
}
__device__ __forceinline__ void st_fold(Pair<double>* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
__device__ __forceinline__ void st_fold(Pair<float>* p, float a, float b) {
  *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

// Chunk tables of one axis in the sweep precision (see chunk_tables()),
// stored once per distinct chunk ("slot").  Two layouts, chosen by the PL
// template flag of the helpers below:
//   PL = false (interleaved): k1, kg [slot][ch][S][2]; kc [chunk][S][4]
//   PL = true  (planar):      k1, kg [slot][ch][2][S]; kc [chunk][4][S]
// In the planar layout the lanes of a warp, which hold consecutive
// densities, read one component of consecutive densities: 8-byte loads of
// contiguous words, one shared-memory wavefront for up to 16 densities,
// where the interleaved slopes and transfer constants sit 16 and 32 bytes
// apart and cost two or three.  Only the FP64 line kernel at full-width
// tiles (16 columns: up to twenty distinct densities of two chunks per warp)
// reads the planar layout (lines_planar()); the row, direct and half-width
// line kernels and the batch tile form read the interleaved one: where a
// warp meets at most eight densities one 16-byte load per entry already
// takes one wavefront, and in the row kernel the extra address arithmetic
// of two planar loads cost more than the wavefronts it saved.
template <typename T>
struct ChunkCoef {
  const T* k1;    // {1/d, a} per point and density
  const T* kg;    // {G, R} per point and density
  const T* kc;    // {P_end, G_start, R_start, 0} per chunk and density
  const int* slot;  // [nc] slot of each chunk of the line
  int ch;
  int nc;
  int tab_elems;  // elements of k1 | kg | kc, contiguous from k1
};

// Copies the chunk tables (k1 | kg | kc, contiguous) and the slot map into
// shared memory once per (persistent) block; returns the shared view.
template <typename T>
__device__ __forceinline__ ChunkCoef<T> stage_tables(const ChunkCoef<T>& g, T* sm_tab,
                                                     int* sm_slot, int tid, int nthreads) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  const int nv = g.tab_elems * (int)sizeof(T) / (int)sizeof(V);
  const V* src = reinterpret_cast<const V*>(g.k1);
  V* dst = reinterpret_cast<V*>(sm_tab);
  for (int i = tid; i < nv; i += nthreads) dst[i] = __ldg(src + i);
  for (int i = tid; i < g.nc; i += nthreads) sm_slot[i] = __ldg(g.slot + i);
  ChunkCoef<T> s = g;
  s.k1 = sm_tab;
  s.kg = sm_tab + (g.kg - g.k1);
  s.kc = sm_tab + (g.kc - g.k1);
  s.slot = sm_slot;
  return s;
}

// This density's rows of chunk c: k1 and kg step 2*S elements per point in
// both layouts.
template <bool SMEM, typename T, bool PL = false>
__device__ __forceinline__ size_t chunk_row(const ChunkCoef<T>& cc, int c, int s, int S) {
  const size_t base = (size_t)ld_one<SMEM>(cc.slot + c) * cc.ch * S * 2;
  return PL ? base + s : base + (size_t)s * 2;
}
// {x, y} components of one (point, density) entry of k1 or kg: the second
// component S elements after the first (planar) or beside it (interleaved).
template <bool SMEM, bool PL, typename T>
__device__ __forceinline__ Pair<T> ld_entry(const T* p, int S) {
  if (PL) return {ld_one<SMEM>(p), ld_one<SMEM>(p + S)};
  return ld_pair<SMEM>(p);
}

template <typename T, typename CT = T>
struct LinesArgs {
  T* p;
  T* out;          // where the solved lines go (p: in place; the map reads p)
  int64_t C;       // contiguous columns per outer block (< 2^31)
  int n;           // points per line
  int64_t ls;      // element stride between points
  int64_t os;      // element stride between outer blocks
  int S;
  uint32_t ctiles;  // ceil(C / W)
  uint32_t tile0;   // tiles tile0 .. ntiles-1 (a slab of outer blocks)
  uint32_t ntiles;  // outer blocks * ctiles
  int box_n;        // rows per TMA box (<= 256)
  int nboxes;       // boxes per tile
  int nchunks;
  ChunkCoef<CT> cc;
  SegList dir_epi;  // (line, chunk) segments, line = (outer*C + col) / S
  int* status;
};

template <typename T, typename CT = T>
struct RowsArgs {
  T* p;
  T* out;  // where the solved rows go (p: in place)
  int64_t rows;  // ny * nz
  int n;         // nx
  int S;
  int R;          // rows per tile
  int64_t pitch;  // shared-memory elements between the rows of a tile
  int64_t tile0;  // tiles tile0 .. ntiles-1 (a slab of rows)
  int64_t ntiles;
  int nchunks;
  int tpc;        // threads per chunk: R*S, or R*S rounded up to a multiple of 32
  ChunkCoef<CT> cc;
  // (row, chunk) segment lists, as for lod_sweep_kernel
  SegList bulk, cells, dir;
  double dt;
  int fuse;
  int* status;
};

// Bytes from the start of dynamic shared memory to its first 128-byte
// boundary.
__device__ __forceinline__ uint32_t smem_pad128(const unsigned char* smem) {
  return (128u - ((uint32_t)__cvta_generic_to_shared(smem) & 127u)) & 127u;
}

// ---- the chunk solve shared by both kernels --------------------------------

// Forward then backward chunk-local passes (zero carries).  k1 points at the
// chunk's first point for this density; consecutive points are 2*S elements
// apart.  Returns the chunk's last forward value (qe) and first backward
// value (x0).  The backward pass reads the slopes a_k again (cheaper than
// holding CH more registers).
template <bool SMEM, typename T, int CH, bool PL = false>
__device__ __forceinline__ void chunk_local(T (&v)[CH], int len, const T* k1, int S, T& qe,
                                            T& x0) {
  T q = T(0);
#pragma unroll
  for (int m = 0; m < CH; ++m) {
    if (m < len) {
      const Pair<T> c = ld_entry<SMEM, PL>(k1 + (size_t)2 * S * m, S);
      q = fma(c.y, q, v[m] * c.x);
      v[m] = q;
    }
  }
  qe = q;
  T x = T(0);
  const int aoff = PL ? S : 1;  // the slope a_k beside 1/d_k
#pragma unroll
  for (int m = CH - 1; m >= 0; --m) {
    if (m < len) {
      x = fma(ld_one<SMEM>(k1 + (size_t)2 * S * m + aoff), x, v[m]);
      v[m] = x;
    }
  }
  x0 = x;
}

// One pass over the chunks of a line: the forward carry into chunk c (cf) and
// the backward carry into it (cb), from every chunk's (qe, x0) pair in shared
// memory (fold columns fw apart) and the chunks' transfer constants.
template <bool SMEM, typename T, bool PL = false>
__device__ __forceinline__ void chunk_carries(const Pair<T>* fold, int fw, int col, int c, int NC,
                                              const ChunkCoef<T>& tab, int s, int S, T& cf_out,
                                              T& cb_out) {
  T cf = T(0), cb = T(0), w = T(1), my = T(0);
  const T* t = tab.kc + (PL ? (size_t)s : (size_t)4 * s);
#pragma unroll 4
  for (int cc = 0; cc < NC; ++cc, t += (size_t)4 * S) {
    // {P_end, G_start} and R_start
    const Pair<T> ag = PL ? Pair<T>{ld_one<SMEM>(t), ld_one<SMEM>(t + S)} : ld_pair<SMEM>(t);
    const T r0 = ld_one<SMEM>(t + (PL ? 2 * S : 2));
    const Pair<T> f = ld_fold(fold + cc * fw + col);  // {qe, x0} of chunk cc
    if (cc == c) my = cf;
    if (cc > c) {
      cb = fma(w, fma(ag.y, cf, f.y), cb);
      w = w * r0;
    }
    cf = fma(ag.x, cf, f.x);
  }
  cf_out = my;
  cb_out = cb;
}

template <bool SMEM, typename T, int CH, bool PL = false>
__device__ __forceinline__ void chunk_fix(T (&v)[CH], int len, const T* kg, int S, T cf, T cb) {
#pragma unroll
  for (int m = 0; m < CH; ++m) {
    if (m < len) {
      const Pair<T> gr = ld_entry<SMEM, PL>(kg + (size_t)2 * S * m, S);
      v[m] = fma(cf, gr.x, fma(cb, gr.y, v[m]));
    }
  }
}

// Self-test of the error path of the bounded waits: one thread initialises a
// barrier that expects one arrival, never arrives, and waits on it with the
// sweeps' wait (limit_ns).  The wait gives up, the kernel records it in
// status as a sweep that gave up would, and returns; no copy was issued, so
// none is in flight.
static __global__ void bounded_wait_selftest_kernel(unsigned long long limit_ns,
                                                    int* __restrict__ status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  tma::mbar_init(&bar, 1);
  tma::fence_barrier_init();
  if (!tma::mbar_wait(&bar, 0, limit_ns)) atomicExch(status, 1);
  tma::mbar_inval(&bar);
}

// Bounded waits for the copies still in flight after a failure, then status.
__device__ __forceinline__ void drain_after_failure(uint64_t* full, int stages, int next_i,
                                                    int outstanding, int* status) {
  for (int j = 0; j < outstanding; ++j) {
    const int i = next_i + j;
    tma::mbar_wait(&full[i % stages], (uint32_t)((i / stages) & 1));
  }
  atomicExch(status, 1);
}

// ---------------------------------------------------------------------------

// Whether the line kernel with W columns reads the planar chunk tables (the
// host passes the matching copy).
constexpr bool lines_planar(int math_bytes, int w) { return math_bytes == 8 && w == 16; }

// MAXNC: the most chunks per line the kernel is compiled for (block of
// W x MAXNC threads).  MAXNC = 8 with 32-point chunks (lines of up to 256
// points) lets the compiler give each thread the registers for its 32 values
// and the chunk tables without spilling.
template <typename T, int CH, int W, int STAGES, bool DIR_EPI, bool SMEM_TAB, int MAXNC,
          typename CT = T>
__global__ void __launch_bounds__(W * MAXNC)
    lod_lines_tma_kernel(const __grid_constant__ CUtensorMap map, const LinesArgs<T, CT> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr bool PL = lines_planar((int)sizeof(CT), W);
  const int NC = blockDim.y;
  const int npad = a.box_n * a.nboxes;
  const size_t stage_elems = (size_t)npad * W;
  // tensor copies need 128-B aligned shared-memory destinations; the pad is
  // added to the shared array itself, so every pointer below stays a
  // shared-memory pointer to the compiler
  T* tiles = reinterpret_cast<T*>(smem_raw + smem_pad128(smem_raw));
  Pair<CT>* fold = reinterpret_cast<Pair<CT>*>(tiles + STAGES * stage_elems);  // 2 x [NC][W]
  uint64_t* full = reinterpret_cast<uint64_t*>(fold + 2 * NC * W);
  CT* sm_tab = reinterpret_cast<CT*>(full + 4);  // chunk tables (SMEM_TAB)
  int* sm_slot = reinterpret_cast<int*>(sm_tab + (SMEM_TAB ? a.cc.tab_elems : 0));

  const int tx = threadIdx.x;
  const int c = threadIdx.y;
  const int tid = c * W + tx;
  const uint32_t stage_bytes = (uint32_t)(stage_elems * sizeof(T));
  const ChunkCoef<CT> tab =
      SMEM_TAB ? stage_tables(a.cc, sm_tab, sm_slot, tid, W * NC) : a.cc;

  if (tid == 0) {
    tma::prefetch_map(&map);
    for (int s = 0; s < STAGES; ++s) tma::mbar_init(&full[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](int st, uint32_t tile) {
    const uint32_t outer = tile / a.ctiles;
    const int col0 = (int)((tile - outer * a.ctiles) * W);
    tma::mbar_arrive_expect_tx(&full[st], stage_bytes);
    for (int b = 0; b < a.nboxes; ++b)
      tma::load_tile_3d(tiles + st * stage_elems + (size_t)b * a.box_n * W, &map, &full[st],
                        col0, b * a.box_n, (int)outer);
  };
  int issued = 0;  // tiles issued by this block (meaningful in thread 0)
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      const uint32_t t = a.tile0 + blockIdx.x + (uint32_t)s * gridDim.x;
      if (t < a.ntiles) {
        issue(s, t);
        ++issued;
      }
    }
  }

  const int S = a.S;
  const int k0 = c * CH;
  const int len = max(0, min(CH, a.n - k0));
  int i = 0;
  for (uint32_t tile = a.tile0 + blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++i) {
    const int st = i % STAGES;
    const bool ok = tma::mbar_wait(&full[st], (uint32_t)((i / STAGES) & 1));
    const uint32_t outer = tile / a.ctiles;
    const uint32_t col = (tile - outer * a.ctiles) * W + tx;
    const bool active = col < (uint32_t)a.C;
    const int lenA = active ? len : 0;
    const int s = (int)(col % (uint32_t)S);
    const T* buf = tiles + st * stage_elems + (size_t)k0 * W + tx;

    CT v[CH];
#pragma unroll
    for (int m = 0; m < CH; ++m) v[m] = (m < lenA) ? (CT)buf[m * W] : CT(0);

    const size_t row = chunk_row<SMEM_TAB, CT, PL>(tab, c, s, S);
    CT qe, x0;
    chunk_local<SMEM_TAB, CT, CH, PL>(v, lenA, tab.k1 + row, S, qe, x0);
    Pair<CT>* sF = fold + (i & 1) * NC * W;
    st_fold(sF + c * W + tx, qe, x0);
    // every thread has read its chunk of this stage: it can be refilled
    if (__syncthreads_or(!ok)) {
      if (tid == 0) drain_after_failure(full, STAGES, i, issued - i, a.status);
      return;
    }
    if (tid == 0) {
      const uint32_t nt = tile + (uint32_t)STAGES * gridDim.x;
      if (nt < a.ntiles) {
        issue(st, nt);
        ++issued;
      }
    }
    CT cf, cb;
    chunk_carries<SMEM_TAB, CT, PL>(sF, W, tx, c, NC, tab, s, S, cf, cb);
    if (lenA == 0) continue;
    chunk_fix<SMEM_TAB, CT, CH, PL>(v, lenA, tab.kg + row, S, cf, cb);
    if (DIR_EPI) {
      const int64_t vcol = (int64_t)outer * a.C + col;
      const int64_t seg = (vcol / S) * a.nchunks + c;
      apply_dirichlet_seg<CT, CH>(v, a.dir_epi, seg, k0, S, s);
    }
    T* ptr = a.out + (int64_t)outer * a.os + col + (int64_t)k0 * a.ls;
#pragma unroll
    for (int m = 0; m < CH; ++m) {
      if (m < lenA) *ptr = (T)v[m];
      ptr += a.ls;
    }
  }
}

// ---------------------------------------------------------------------------

// Blocks of up to 256 threads with chunks of up to 16 points are compiled for
// two resident blocks per SM (the plan sizes their shared memory for two).
constexpr int rows_min_blocks(int ch, int maxt) { return (ch <= 16 && maxt <= 256) ? 2 : 1; }

// MINB: resident blocks per SM the kernel is compiled for (two at 32-point
// chunks caps the registers at 128: more warps, some spilled state).
// SC > 0: a build for exactly SC densities (a.S == SC), so that every offset
// along a row (stage, tables, stores: multiples of S) is a compile-time
// constant; PLR: that build reading the planar chunk tables.
template <typename T, int CH, int STAGES, bool SMEM_TAB, int MAXT, typename CT = T,
          int MINB = rows_min_blocks(CH, MAXT), int SC = 0, bool PLR = false>
__global__ void __launch_bounds__(MAXT, MINB)
    lod_rows_tma_kernel(const RowsArgs<T, CT> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // Threads: column (r, s) fastest, then chunk c.  A stage holds R rows at a
  // padded pitch (pitch = S mod 16 elements), so the lanes of a warp, which
  // read consecutive columns, hit consecutive banks.
  const int S = SC > 0 ? SC : a.S;
  const int n = a.n;
  const int R = a.R;
  const int FW = R * S;  // columns per tile
  const int NC = a.nchunks;
  const size_t pitch = a.pitch;
  const size_t row_elems = (size_t)n * S;
  const size_t stage_elems = pitch * R;
  // 128-B aligned stages; the pad is added to the shared array itself, so
  // every pointer below stays a shared-memory pointer to the compiler
  const uint32_t pad = smem_pad128(smem_raw);
  T* tiles = reinterpret_cast<T*>(smem_raw + pad);
  Pair<CT>* fold = reinterpret_cast<Pair<CT>*>(tiles + STAGES * stage_elems);  // 2 x [NC][FW]
  const size_t full_off =
      (pad + (STAGES * stage_elems * sizeof(T) + 2 * NC * FW * sizeof(Pair<CT>)) + 15) &
      ~(size_t)15;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + full_off);
  CT* sm_tab = reinterpret_cast<CT*>(full + 4);  // chunk tables (SMEM_TAB)
  int* sm_slot = reinterpret_cast<int*>(sm_tab + (SMEM_TAB ? a.cc.tab_elems : 0));

  const int tid = threadIdx.x;
  const int nthreads = blockDim.x;
  // a.tpc threads per chunk (FW, or FW rounded up to whole warps so that the
  // lanes of a warp read one chunk: lanes of two chunks 32*CH*S elements
  // apart would meet on the same banks); lanes past FW idle
  const int fc = tid % a.tpc;  // column in the tile
  const int c = tid / a.tpc;   // chunk
  const int r = fc / S;
  const int s = fc - r * S;
  const int k0 = c * CH;
  const int len = (c < NC) ? max(0, min(CH, n - k0)) : 0;
  const ChunkCoef<CT> tab =
      SMEM_TAB ? stage_tables(a.cc, sm_tab, sm_slot, tid, nthreads) : a.cc;
  if (tid == 0) {
    for (int st = 0; st < STAGES; ++st) tma::mbar_init(&full[st], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  const size_t crow = (c < NC) ? chunk_row<SMEM_TAB, CT, PLR>(tab, c, s, S) : 0;
  const CT* k1 = tab.k1 + crow;
  const CT* kg = tab.kg + crow;

  auto tile_rows = [&](int64_t tile) -> int {
    return (int)min((int64_t)R, a.rows - tile * R);
  };
  auto issue = [&](int st, int64_t tile) {
    const int nr = tile_rows(tile);
    const uint32_t rb = (uint32_t)(row_elems * sizeof(T));
    tma::mbar_arrive_expect_tx(&full[st], rb * nr);
    for (int q = 0; q < nr; ++q)
      tma::load_bulk(tiles + st * stage_elems + q * pitch, a.p + (tile * R + q) * row_elems, rb,
                     &full[st]);
  };
  int issued = 0;
  if (tid == 0) {
    for (int st = 0; st < STAGES; ++st) {
      const int64_t t = a.tile0 + blockIdx.x + (int64_t)st * gridDim.x;
      if (t < a.ntiles) {
        issue(st, t);
        ++issued;
      }
    }
  }

  int i = 0;
  for (int64_t tile = a.tile0 + blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++i) {
    const int st = i % STAGES;
    const bool ok = tma::mbar_wait(&full[st], (uint32_t)((i / STAGES) & 1));
    const int nr = tile_rows(tile);
    const int64_t row = tile * R + r;
    const int lenA = (r < nr) ? len : 0;
    const T* rb = tiles + st * stage_elems + r * pitch + (size_t)k0 * S + s;
    CT v[CH];
#pragma unroll
    for (int m = 0; m < CH; ++m) v[m] = (m < lenA) ? (CT)rb[m * S] : CT(0);

    // ---- prologue in registers: bulk -> cells -> Dirichlet for this chunk
    const int64_t seg = row * NC + c;
    if (lenA > 0 && (a.fuse & (kFuseBulk | kFuseCells | kFuseDirPro))) {
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
        // agents sorted by (voxel, list order); one voxel's agents accumulate
        // in FP64 before rounding
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
      if (a.fuse & kFuseDirPro) apply_dirichlet_seg<CT, CH>(v, a.dir, seg, k0, S, s);
    }

    // ---- sweep
    CT qe, x0;
    chunk_local<SMEM_TAB, CT, CH, PLR>(v, lenA, k1, S, qe, x0);
    Pair<CT>* sF = fold + (i & 1) * NC * FW;
    if (c < NC && fc < FW) st_fold(sF + c * FW + fc, qe, x0);
    // every thread has its chunk in registers: the stage can be refilled
    if (__syncthreads_or(!ok)) {
      if (tid == 0) drain_after_failure(full, STAGES, i, issued - i, a.status);
      return;
    }
    if (tid == 0) {
      const int64_t nt = tile + (int64_t)STAGES * gridDim.x;
      if (nt < a.ntiles) {
        issue(st, nt);
        ++issued;
      }
    }
    if (lenA == 0) continue;
    CT cf, cb;
    chunk_carries<SMEM_TAB, CT, PLR>(sF, FW, fc, c, NC, tab, s, S, cf, cb);
    chunk_fix<SMEM_TAB, CT, CH, PLR>(v, lenA, kg, S, cf, cb);
    // ---- epilogue: Dirichlet before the next axis
    if (a.fuse & kFuseDirEpi) apply_dirichlet_seg<CT, CH>(v, a.dir, seg, k0, S, s);
    // straight to global memory: the lanes of a warp write the S densities of
    // consecutive rows at one point
    T* out = a.out + row * (int64_t)row_elems + (int64_t)k0 * S + s;
#pragma unroll
    for (int m = 0; m < CH; ++m)
      if (m < lenA) out[(int64_t)m * S] = (T)v[m];
  }
}

// ---------------------------------------------------------------------------
// Sweeps without shared-memory staging of the field (any axis).  Columns are
// the (line, density) pairs numbered as in lod_sweep_kernel: vcol = outer*C +
// col, so consecutive threads of a warp read consecutive addresses for y and
// z, and the S densities of consecutive rows for x.  Each block solves W
// columns x n points; every thread loads its chunk straight from global
// memory (up to CH loads in flight per thread), the chunk tables are read
// through L1 (little shared memory is used, so L1 keeps its capacity), and
// for x the rest of the step (bulk, cells, Dirichlet) is applied to the
// chunk in registers before the sweep.

template <typename T, typename CT = T>
struct DirectArgs {
  T* p;
  T* out;                // where the solved lines go (p: in place)
  int64_t col0;          // first column of this launch (a slab of planes)
  int64_t ncols;         // end of the launch's (line, density) columns
  int64_t C;             // columns per outer block
  int64_t outer_stride;  // elements
  int64_t line_stride;   // elements between points of a line
  int n;
  int nchunks;
  int S;
  ChunkCoef<CT> cc;
  SegList bulk, cells, dir_pro, dir_epi;
  double dt;
  int fuse;
};

template <typename T, int CH, int W, int MODE, typename CT = T>
__global__ void __launch_bounds__(512) lod_sweep_direct_kernel(const DirectArgs<T, CT> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int NC = blockDim.y;
  Pair<CT>* fold = reinterpret_cast<Pair<CT>*>(smem_raw);  // [NC][W]
  // this block's copy of the per-chunk constants and the slot map
  CT* kc_sm = reinterpret_cast<CT*>(fold + NC * W);        // [NC][S][4]
  int* slot_sm = reinterpret_cast<int*>(kc_sm + (size_t)4 * NC * a.S);
  const int tx = threadIdx.x;
  const int c = threadIdx.y;
  {
    const int tid = c * W + tx, nt = W * NC;
    for (int i = tid; i < 4 * NC * a.S; i += nt) kc_sm[i] = __ldg(a.cc.kc + i);
    for (int i = tid; i < NC; i += nt) slot_sm[i] = __ldg(a.cc.slot + i);
  }
  const int S = a.S;
  const int k0 = c * CH;
  const int64_t vcol = a.col0 + (int64_t)blockIdx.x * W + tx;
  const bool active = vcol < a.ncols;
  const int lenA = active ? max(0, min(CH, a.n - k0)) : 0;
  int s = 0;
  T* ptr = a.p;
  int64_t seg = 0;
  if (active) {
    const int64_t outer = vcol / a.C;
    const int64_t col = vcol - outer * a.C;
    s = (int)(col % S);
    ptr = a.p + outer * a.outer_stride + col + (int64_t)k0 * a.line_stride;
    seg = (vcol / S) * a.nchunks + c;
  }
  const int64_t ls = a.line_stride;

  CT v[CH];
  {
    const T* q = ptr;
#pragma unroll
    for (int m = 0; m < CH; ++m) {
      v[m] = (m < lenA) ? (CT)*q : CT(0);
      q += ls;
    }
  }

  if (MODE == kSweepFull && lenA > 0) {
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
      // agents sorted by (voxel, list order); one voxel's agents accumulate
      // in FP64 before rounding
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

  __syncthreads();  // kc_sm, slot_sm
  ChunkCoef<CT> tab = a.cc;
  tab.kc = kc_sm;
  tab.slot = slot_sm;
  const size_t row = active ? ((size_t)slot_sm[c] * tab.ch * S + s) * 2 : 0;
  CT qe, x0;
  chunk_local<false, CT, CH>(v, lenA, a.cc.k1 + row, S, qe, x0);
  st_fold(fold + c * W + tx, qe, x0);
  __syncthreads();
  CT cf, cb;
  chunk_carries<true, CT>(fold, W, tx, c, NC, tab, s, S, cf, cb);
  if (lenA == 0) return;
  chunk_fix<false, CT, CH>(v, lenA, a.cc.kg + row, S, cf, cb);
  if (MODE != kSweepPlain && (a.fuse & kFuseDirEpi))
    apply_dirichlet_seg<CT, CH>(v, a.dir_epi, seg, k0, S, s);
  T* dst = a.out + (ptr - a.p);
#pragma unroll
  for (int m = 0; m < CH; ++m) {
    if (m < lenA) *dst = (T)v[m];
    dst += ls;
  }
}

}  // namespace bfvm
