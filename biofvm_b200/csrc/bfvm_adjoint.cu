// Reverse-mode derivative of n transport steps (libbfvm.so, FP64).
//
// bfvm_adjoint_forward runs n steps exactly as bfvm_step does and keeps the
// field at every k-th step (checkpoints).  bfvm_adjoint_backward takes the
// derivative of a loss with respect to the final field (the seed) and walks
// the steps backwards: per segment of k steps it recomputes the segment from
// its checkpoint, keeping the output of every solve (3 fields per step), and
// then applies the adjoint of each step in reverse order (adjoint solves are
// the forward sweeps: the LOD matrices are symmetric; the Dirichlet overwrite
// becomes a zeroing; the bulk and cell updates are differentiated in place,
// bfvm_adjoint_kernels.cuh).  It returns the derivatives with respect to
// every substrate's diffusion coefficient and decay rate, every agent's
// temp1/temp2 constants (BioFVM_basic_agent.cpp:139-147; the chain rule to
// secretion/uptake rates is the caller's, they are plain products) and the
// initial field.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "bfvm.h"
#include "bfvm_adjoint_kernels.cuh"
#include "bfvm_state.h"

namespace bfvm_rt {

struct AdjointTape {
  bool valid = false;
  double dt = 0;
  int nsteps = 0, flags = 0, k = 1;
  int S = 0;
  int64_t N = 0, agents = 0, bulk = 0, nodes = 0;
  DevBuf ckpt, tape, abar, part, acc, gt1, gt2;
};

void adjoint_release(bfvm_solver* m) {
  delete m->adj;
  m->adj = nullptr;
}

namespace {

using namespace bfvm;

// Runs the solver's kernels on another FP64 field of the same shape.
struct FieldSwap {
  bfvm_solver* m;
  DevBuf saved;
  FieldSwap(bfvm_solver* mm, void* ptr) : m(mm), saved(mm->p) {
    m->p.ptr = ptr;
    m->p.bytes = saved.bytes;
  }
  ~FieldSwap() {
    m->p = saved;
    saved.ptr = nullptr;
  }
  FieldSwap(const FieldSwap&) = delete;
  FieldSwap& operator=(const FieldSwap&) = delete;
};

size_t field_bytes(const bfvm_solver* m) { return (size_t)m->NS() * sizeof(double); }
// stride of the stored fields: 256-byte aligned, as the TMA sweeps want
size_t field_stride(const bfvm_solver* m) { return (field_bytes(m) + 255) / 256 * 256; }

void copy_field(bfvm_solver* m, void* dst, const void* src) {
  BFVM_CUDA(cudaMemcpyAsync(dst, src, field_bytes(m), cudaMemcpyDeviceToDevice, m->stream));
}

// Sweeps write to another field while it is alive (out-of-place solves).
struct OutSwap {
  bfvm_solver* m;
  OutSwap(bfvm_solver* mm, void* out) : m(mm) { m->sweep_out = out; }
  ~OutSwap() { m->sweep_out = nullptr; }
  OutSwap(const OutSwap&) = delete;
  OutSwap& operator=(const OutSwap&) = delete;
};

// One forward step on the current field with every solve output kept:
// x, y, z receive the field after the x, y and z solves.
void step_keeping_solves(bfvm_solver* m, double dt, int flags, const void* in, unsigned char* x,
                         unsigned char* y, unsigned char* z) {
  copy_field(m, x, in);
  {
    FieldSwap f(m, x);
    if (flags & BFVM_STEP_BULK) bulk_any(m, dt);
    if (flags & BFVM_STEP_CELLS) cells_any(m);
    if (!(flags & BFVM_STEP_DIFFUSION)) {
      copy_field(m, z, x);
      return;
    }
    dirichlet_standalone<double>(m);
    sweep(m, 0, 0, dt);
  }
  if (m->dir_unique == 0) {
    // no Dirichlet node to overwrite between the solves: the y and z solves
    // read the previous solve's output and write the next slot (no copies)
    {
      FieldSwap f(m, x);
      OutSwap o(m, y);
      sweep(m, 1, 0, dt);
    }
    FieldSwap f(m, y);
    OutSwap o(m, z);
    sweep(m, 2, 0, dt);
    return;
  }
  copy_field(m, y, x);
  {
    FieldSwap f(m, y);
    dirichlet_standalone<double>(m);
    sweep(m, 1, 0, dt);
  }
  copy_field(m, z, y);
  {
    FieldSwap f(m, z);
    dirichlet_standalone<double>(m);
    sweep(m, 2, 0, dt);
  }
}

// Blocks of the dot-product passes (the same for every solve of a run, so
// their partial sums can accumulate in place).
int dot_blocks(const bfvm_solver* m) {
  const int64_t rows = (int64_t)m->ny * m->nz;
  return (int)std::max<int64_t>(1, std::min<int64_t>(8 * m->num_sms, rows));
}

// Adds this solve's -a.(L y) and -a.y partial sums to T.part.
void dot_into_part(bfvm_solver* m, AdjointTape& T, const double* y, int axis) {
  const int S = m->S;
  const int threads = S * std::max(1, 256 / S);  // a multiple of S (S <= 256)
  const size_t smem = 2 * sizeof(double) * (size_t)threads;
  adj_axis_dot_kernel<<<dot_blocks(m), threads, smem, m->stream>>>(
      T.abar.as<double>(), y, m->nx, m->ny, m->nz, S, axis, T.part.as<double>());
  check_launch(m);
}

void zero_nodes(bfvm_solver* m, AdjointTape& T) {
  if (m->dir_unique == 0) return;
  const int64_t work = m->dir_unique * m->S;
  adj_zero_nodes_kernel<<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
      T.abar.as<double>(), m->S, m->dir_unique, m->d_dir_vox.as<int64_t>());
  check_launch(m);
}

void adjoint_forward(bfvm_solver* m, double dt, int nsteps, int flags, int k) {
  require(m->precision == BFVM_FP64, "the adjoint runs in FP64 only");
  require(nsteps >= 1, "nsteps must be positive");
  require(k >= 1, "checkpoint interval must be positive");
  require((flags & ~BFVM_STEP_ALL) == 0, "unknown step flags");
  require(m->S <= 256, "the adjoint supports at most 256 densities");
  require(m->nx <= 1024 && m->ny <= 1024 && m->nz <= 1024,
          "the adjoint supports lines of at most 1024 points");
  check_lod_mesh(m);
  if (!m->adj) m->adj = new AdjointTape;
  AdjointTape& T = *m->adj;
  T.valid = false;
  if (!m->setup_done) thomas_setup(m, dt);
  build_all(m);
  const size_t F = field_stride(m);
  const int ncp = (nsteps + k - 1) / k;
  T.ckpt.ensure((size_t)ncp * F);
  for (int t = 0; t < nsteps; ++t) {
    if (t % k == 0) copy_field(m, T.ckpt.as<unsigned char>() + (size_t)(t / k) * F, m->p.ptr);
    if (flags & BFVM_STEP_DIFFUSION) {
      step_once(m, dt, flags, nullptr);
    } else {
      if (flags & BFVM_STEP_BULK) bulk_any(m, dt);
      if (flags & BFVM_STEP_CELLS) cells_any(m);
    }
  }
  check_status(m);
  T.dt = dt;
  T.nsteps = nsteps;
  T.flags = flags;
  T.k = k;
  T.S = m->S;
  T.N = m->N();
  T.agents = m->n_agents;
  T.bulk = (int64_t)m->bulk_vox.size();
  T.nodes = m->dir_unique;
  T.valid = true;
}

void adjoint_backward(bfvm_solver* m, const double* seed, int seed_on_device, double* grad_D,
                      double* grad_decay, double* grad_t1, double* grad_t2, double* grad_p0) {
  require(m->adj && m->adj->valid, "no recorded forward run (bfvm_adjoint_forward)",
          BFVM_ERR_STATE);
  AdjointTape& T = *m->adj;
  require(seed != nullptr, "null seed");
  build_all(m);
  require(T.S == m->S && T.N == m->N() && T.agents == m->n_agents &&
              T.bulk == (int64_t)m->bulk_vox.size() && T.nodes == m->dir_unique && m->setup_done,
          "the solver changed since bfvm_adjoint_forward", BFVM_ERR_STATE);
  const int S = m->S;
  const int64_t A = m->n_agents;
  const double dt = T.dt;
  const int flags = T.flags, k = T.k;
  const size_t F = field_stride(m), FB = field_bytes(m);
  cudaStream_t st = m->stream;

  T.abar.ensure(F);
  BFVM_CUDA(cudaMemcpyAsync(T.abar.ptr, seed, FB,
                            seed_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            st));
  T.acc.ensure(2 * S * sizeof(double));
  BFVM_CUDA(cudaMemsetAsync(T.acc.ptr, 0, 2 * S * sizeof(double), st));
  const int dblocks = dot_blocks(m);
  T.part.ensure((size_t)dblocks * 2 * S * sizeof(double));
  BFVM_CUDA(cudaMemsetAsync(T.part.ptr, 0, (size_t)dblocks * 2 * S * sizeof(double), st));
  if (A > 0) {
    T.gt1.ensure((size_t)A * S * sizeof(double));
    T.gt2.ensure((size_t)A * S * sizeof(double));
    BFVM_CUDA(cudaMemsetAsync(T.gt1.ptr, 0, (size_t)A * S * sizeof(double), st));
    BFVM_CUDA(cudaMemsetAsync(T.gt2.ptr, 0, (size_t)A * S * sizeof(double), st));
  }
  const int seg_len = std::min(k, T.nsteps);
  T.tape.ensure((size_t)3 * seg_len * F);
  unsigned char* tape = T.tape.as<unsigned char>();
  auto tx = [&](int j) { return tape + (size_t)(3 * j) * F; };
  auto ty = [&](int j) { return tape + (size_t)(3 * j + 1) * F; };
  auto tz = [&](int j) { return tape + (size_t)(3 * j + 2) * F; };

  const int nseg = (T.nsteps + k - 1) / k;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int t0 = seg * k, len = std::min(T.nsteps, t0 + k) - t0;
    const unsigned char* ck = T.ckpt.as<unsigned char>() + (size_t)seg * F;
    for (int j = 0; j < len; ++j)
      step_keeping_solves(m, dt, flags, j == 0 ? ck : tz(j - 1), tx(j), ty(j), tz(j));
    for (int j = len - 1; j >= 0; --j) {
      if (flags & BFVM_STEP_DIFFUSION) {
        const unsigned char* ys[3] = {tx(j), ty(j), tz(j)};
        for (int ax = 2; ax >= 0; --ax) {
          {
            FieldSwap f(m, T.abar.ptr);
            sweep(m, ax, 0, dt);
          }
          dot_into_part(m, T, reinterpret_cast<const double*>(ys[ax]), ax);
          zero_nodes(m, T);
        }
      }
      const double* in = reinterpret_cast<const double*>(j == 0 ? ck : tz(j - 1));
      const bool bulk = (flags & BFVM_STEP_BULK) && T.bulk > 0;
      if ((flags & BFVM_STEP_CELLS) && A > 0) {
        adj_cells_kernel<<<(unsigned)blocks_for(A * S, 256), 256, 0, st>>>(
            T.abar.as<double>(), in, S, A, m->d_ag_key.as<uint64_t>(), m->d_ag_idx.as<int>(),
            m->d_ag_t1.as<double>(), m->d_ag_t2.as<double>(), bulk ? T.bulk : 0,
            m->d_bulk_vox.as<int64_t>(), m->d_bulk_st.as<double>(), m->d_bulk_su.as<double>(), dt,
            T.gt1.as<double>(), T.gt2.as<double>());
        check_launch(m);
      }
      if (bulk) {
        adj_bulk_kernel<<<(unsigned)blocks_for(T.bulk * S, 256), 256, 0, st>>>(
            T.abar.as<double>(), S, T.bulk, m->d_bulk_vox.as<int64_t>(),
            m->d_bulk_su.as<double>(), dt);
        check_launch(m);
      }
    }
  }
  if (flags & BFVM_STEP_DIFFUSION) {
    adj_reduce_parts_kernel<<<2 * S, kAdjReduceThreads, 0, st>>>(T.part.as<double>(), dblocks,
                                                                  S, T.acc.as<double>());
    check_launch(m);
  }
  std::vector<double> acc(2 * S);
  BFVM_CUDA(cudaMemcpyAsync(acc.data(), T.acc.ptr, acc.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  if (A > 0 && grad_t1)
    BFVM_CUDA(cudaMemcpyAsync(grad_t1, T.gt1.ptr, (size_t)A * S * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  if (A > 0 && grad_t2)
    BFVM_CUDA(cudaMemcpyAsync(grad_t2, T.gt2.ptr, (size_t)A * S * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  if (grad_p0) BFVM_CUDA(cudaMemcpyAsync(grad_p0, T.abar.ptr, FB, cudaMemcpyDeviceToHost, st));
  BFVM_CUDA(cudaStreamSynchronize(st));
  check_status(m);
  // c1 = dt D / dx / dx and c2 = dt decay / 3 (BioFVM_solvers.cpp:111-119)
  for (int s = 0; s < S; ++s) {
    if (grad_D) grad_D[s] = acc[s] * (dt / m->dx / m->dx);
    if (grad_decay) grad_decay[s] = acc[S + s] * (dt / 3.0);
  }
}

}  // namespace
}  // namespace bfvm_rt

using namespace bfvm_rt;

extern "C" {

int bfvm_adjoint_forward(bfvm_solver* m, double dt, int nsteps, int flags, int checkpoint_every) {
  return SOLVER_CALL(m, adjoint_forward(m, dt, nsteps, flags, checkpoint_every));
}

int bfvm_adjoint_backward(bfvm_solver* m, const double* seed, int seed_on_device, double* grad_D,
                          double* grad_decay, double* grad_temp1, double* grad_temp2,
                          double* grad_p0) {
  return SOLVER_CALL(m, adjoint_backward(m, seed, seed_on_device, grad_D, grad_decay, grad_temp1,
                                         grad_temp2, grad_p0));
}

int bfvm_adjoint_release(bfvm_solver* m) { return SOLVER_CALL(m, adjoint_release(m)); }

}  // extern "C"
