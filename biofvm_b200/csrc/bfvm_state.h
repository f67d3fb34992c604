// Internal to libbfvm.so: the solver state and the host helpers shared by
// the translation units of the library (the single-instance C ABI in
// bfvm_solver.cu, the batched instances in bfvm_batch.cu).  Not installed.
#pragma once

#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfvm.h"
#include "bfvm_kernels.cuh"

namespace bfvm_rt {


extern thread_local std::string g_last_error;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define BFVM_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw Error(e_ == cudaErrorMemoryAllocation ? BFVM_ERR_NOMEM : BFVM_ERR_CUDA,       \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

inline void require(bool ok, const std::string& msg, int code = BFVM_ERR_ARG) {
  if (!ok) throw Error(code, msg);
}

// A growable device allocation.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  void ensure(size_t nbytes) {
    if (nbytes <= bytes && ptr) return;
    release();
    if (nbytes == 0) return;
    BFVM_CUDA(cudaMalloc(&ptr, nbytes));
    bytes = nbytes;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

template <typename T>
void upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty())
    BFVM_CUDA(cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

// Device copy of a segment list (see SegList in bfvm_kernels.cuh).
struct DevSegList {
  DevBuf off, pos, a, b;
  bool present = false;
  bfvm::SegList view() const {
    bfvm::SegList L;
    L.off = off.as<int>();
    L.pos = pos.as<int>();
    L.a = a.as<double>();
    L.b = b.as<double>();
    return L;
  }
  void release() {
    off.release();
    pos.release();
    a.release();
    b.release();
    present = false;
  }
};

struct Axis {
  int ch = 16;  // points per thread
  int tw = 32;  // columns per block
  int minb = 1; // resident blocks per SM the kernel is compiled for (1 or 2)
  int kind = 0; // kernel under BFVM_PATH_AUTO: 0 = default, else a BFVM_PATH_* value
  int stages = 0;  // x row kernel: tiles in its shared-memory ring (0 = 2)
  int build = 2;   // x row kernel: 0 any density count, 1 a build for this
                   // density count, 2 the same reading planar tables
                   // (bfvm_set_row_build; 2 runs where it applies)
  bool user = false;  // set through bfvm_set_sweep_config or the tuner
};

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return BFVM_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return BFVM_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return BFVM_ERR_STATE;
  }
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) BFVM_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

inline int64_t blocks_for(int64_t work, int threads) { return (work + threads - 1) / threads; }

}  // namespace bfvm_rt

namespace bfvm_rt {
struct AdjointTape;
}

struct bfvm_solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;

  // mesh (Cartesian_Mesh, BioFVM_mesh.h:146-188)
  int nx = 1, ny = 1, nz = 1;
  double dx = 1, dy = 1, dz = 1, dV = 1;
  double bbox[6] = {-0.5, -0.5, -0.5, 0.5, 0.5, 0.5};
  bool uniform = true;

  // densities
  int S = 1;
  std::vector<double> D{0.0}, decay{0.0};
  int precision = BFVM_FP64;
  bfvm_rt::DevBuf p;

  // Thomas coefficients (computed once, BioFVM_solvers.cpp:87,172), with the
  // dt and coefficients they were computed from
  bool setup_done = false;
  double setup_dt = 0.0;
  std::vector<double> setup_D, setup_decay;
  bfvm_rt::DevBuf coef[3];  // per axis: inv_den, fwd, bwd [n*S] then c1 [S], in the sweep precision
  std::vector<double> h_c1[3], h_den[3], h_cx[3];  // FP64 host copies per axis
  bfvm_rt::DevBuf chunk[3];     // per axis: chunk tables k1, kg, kc by slot (sweep precision),
                                // planar layout (FP64 line kernel at 16-column tiles)
  bfvm_rt::DevBuf chunk_il[3];  // the same tables interleaved (every other kernel)
  bfvm_rt::DevBuf chunk_slots[3];  // per axis: slot of every chunk
  int chunk_ch[3] = {0, 0, 0};
  int chunk_nslots[3] = {0, 0, 0};
  bfvm_rt::Axis axis[3];

  // bulk sources/sinks: non-identity voxels, ascending
  std::vector<int64_t> bulk_vox;
  std::vector<double> bulk_st, bulk_su;
  bool bulk_dirty = true;
  bfvm_rt::DevBuf d_bulk_vox, d_bulk_st, d_bulk_su;
  // the same list with its coefficient rows shared: voxel and row index
  // (int32) per listed voxel, unique (S*T, U+S) rows [rows][S][2]; used by
  // the stand-alone bulk kernel when the rows compress (bulk_rows > 0)
  int64_t bulk_rows = 0;
  bfvm_rt::DevBuf d_bulk_vox32, d_bulk_row, d_bulk_tab;
  bfvm_rt::DevSegList seg_bulk;

  // Dirichlet nodes in insertion order (BioFVM_microenvironment.h:102-103)
  std::vector<int64_t> dir_vox;
  std::vector<double> dir_val;
  bool dir_dirty = true;
  int64_t dir_unique = 0;
  std::vector<int64_t> dir_sorted;  // the unique nodes as uploaded (ascending)
  bfvm_rt::DevBuf d_dir_vox, d_dir_val;
  bfvm_rt::DevSegList seg_dir_x, seg_dir_y;

  // Agents, held on the device only: voxel[A], temp1[A][S], temp2[A][S] in
  // list order, and the list order stably sorted by voxel (key = voxel,
  // idx = position in the list), rebuilt on the device when the agents change.
  int64_t n_agents = 0;
  bool ag_dirty = true;      // sorted order out of date
  bool ag_seg_dirty = true;  // segment lists of the fused x prologue out of date
  bfvm_rt::DevBuf d_ag_vox_orig, d_ag_t1, d_ag_t2;
  bfvm_rt::DevBuf d_ag_key, d_ag_idx_in, d_ag_idx, d_sort_tmp;
  bfvm_rt::DevBuf d_gather;
  bfvm_rt::DevSegList seg_cells;
  // Asynchronous agent exchange (bfvm_set_agents_async,
  // bfvm_get_agent_densities_async), set up on first use: uploads and their
  // sort run on xf_up into the spare buffer set, which then swaps with the
  // current one; reads of d_gather go out on xf_down.  Events: xf_up_done
  // (spare set filled and sorted), xf_spare_free (compute work that read the
  // spare set, recorded when it stopped being current), xf_gathered
  // (d_gather written), xf_down_done (d_gather copied out).
  cudaStream_t xf_up = nullptr, xf_down = nullptr;
  cudaEvent_t xf_up_done = nullptr, xf_spare_free = nullptr, xf_gathered = nullptr,
              xf_down_done = nullptr;
  bool xf_spare_recorded = false, xf_up_pending = false, xf_down_pending = false;
  bfvm_rt::DevBuf xf_vox, xf_t1, xf_t2, xf_key, xf_idx_in, xf_idx, xf_sort_tmp;

  // device status word: set to non-zero by a kernel whose bounded wait failed
  bfvm_rt::DevBuf d_status;
  int num_sms = 148;
  int path = 0;  // BFVM_PATH_*
  int fuse_sources = 0;  // bulk/cell updates in the x sweep's prologue
  int lod_dims = 3;      // 2 while a LOD_2D step runs: sweeps of the z = 0 plane only
  int slab_planes = 0;   // x and y sweeps by slabs of this many z planes (0: whole field)
  void* sweep_out = nullptr;  // sweeps write here instead of in place (the adjoint's recompute)
  // whole steps of a small field in one thread-block cluster (bfvm_step under
  // BFVM_PATH_AUTO): enabled flag, and the FP64 Thomas tables it reads per
  // axis (den [n][S], cx [n][S], c1 [S]), rebuilt after each Thomas setup
  int cluster_steps = 0;
  bool cl_tab_ok = false;
  bfvm_rt::DevBuf cl_tab[3];
  // whole steps of a small field in one cooperative launch over all SMs
  // (bfvm_step under BFVM_PATH_AUTO, on by default): enabled flag, the per-call
  // scratch (Dirichlet values and line masks, bulk and agent voxel maps), and
  // the kernels' resident blocks per SM (0: not queried yet)
  int grid_steps = 1;
  bfvm_rt::DevBuf d_grid_maps;
  // the device lists change: every rebuild of the bulk, Dirichlet or agent
  // lists counts one; the grid-steps maps keep the count they were built at
  int64_t lists_version = 0;
  int64_t grid_maps_version = -1;
  int grid_maps_S = 0;
  int grid_per_sm[2] = {0, 0};  // 4- and 8-point chunk kernels (-1: not usable)
  // cached tensor maps of the line sweeps, per axis, with the geometry they
  // were encoded for (field address, element size, C, n, outer blocks, the
  // two strides, tile width, box rows): a resize that keeps the allocation,
  // a precision change or a LOD_2D step re-encodes them
  CUtensorMap maps[3];
  int64_t map_geom[3][9] = {};

  // z slab of a field split by z planes over several solvers (one per GPU):
  // this solver holds global planes [zs_bounds[zs_rank], zs_bounds[zs_rank+1])
  // of zs_bounds[zs_ranks] planes (zs_ranks = 0: not split).  Its z sweep
  // uses the global line's Thomas rows for its planes; bfvm_zslab_fixup
  // joins the slabs with the per-density constants of every slab
  // (zs_const [ranks][S][3]: P, Gs, R) and of its own planes
  // (zs_pt [nz][S][2]: G, Rk), built with the Thomas set-up.
  int zs_ranks = 0, zs_rank = 0;
  std::vector<int> zs_bounds;
  bfvm_rt::DevBuf zs_const, zs_pt;

  // gradient vectors [N][S][3] FP64 (allocated and zeroed on first use)
  bfvm_rt::DevBuf d_grad;

  // checkpoints and buffers of the adjoint (bfvm_adjoint.cu), when used
  bfvm_rt::AdjointTape* adj = nullptr;

  int64_t N() const { return (int64_t)nx * ny * nz; }
  int64_t NS() const { return N() * S; }
  size_t elem() const { return precision == BFVM_FP64 ? sizeof(double) : sizeof(float); }
  // element size of the sweeps' arithmetic and coefficient tables
  size_t math_elem() const { return precision == BFVM_FP32 ? sizeof(float) : sizeof(double); }
};

namespace bfvm_rt {

inline void check_launch(bfvm_solver* m) {
  m->launches++;
  BFVM_CUDA(cudaGetLastError());
}

template <typename T>
bfvm::AxisCoef<T> coef_view(const bfvm_solver* m, int a) {
  const int ns[3] = {m->nx, m->ny, m->nz};
  const size_t nS = (size_t)ns[a] * m->S;
  const T* base = m->coef[a].as<T>();
  bfvm::AxisCoef<T> c;
  c.inv_den = base;
  c.fwd = base + nS;
  c.bwd = base + 2 * nS;
  c.c1 = base + 3 * nS;
  return c;
}

// Defined in bfvm_solver.cu.
void thomas_setup(bfvm_solver* m, double dt);
void build_all(bfvm_solver* m);
void check_lod_mesh(bfvm_solver* m);
void check_status(bfvm_solver* m);
void step_once(bfvm_solver* m, double dt, int flags, cudaEvent_t* ev);
void sweep(bfvm_solver* m, int ax, int fuse, double dt, int64_t z0 = 0, int64_t z1 = -1);
void tune_sweeps(bfvm_solver* m, double dt, int reps);
void bulk_any(bfvm_solver* m, double dt);
void cells_any(bfvm_solver* m);
template <typename T>
void dirichlet_standalone(bfvm_solver* m);
// Defined in bfvm_adjoint.cu.
void adjoint_release(bfvm_solver* m);

}  // namespace bfvm_rt

#define SOLVER_CALL(m, ...)                                     \
  guarded([&] {                                                 \
    require((m) != nullptr, "null solver handle");              \
    DeviceGuard dg_((m)->device);                               \
    __VA_ARGS__;                                                \
  })
