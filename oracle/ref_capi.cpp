// Test infrastructure only: a C-ABI harness that drives the UNMODIFIED BioFVM
// reference (compiled from its own sources into oracle/_ref/) so that Python
// tests, the golden-fixture generator and the CPU baseline arm of bench.py can
// run the reference's own code on seeded synthetic scenarios.
//
// Nothing in the product links this file.  It is the checker / baseline.
//
// Harness-side fixes the reference needs to run at all (none edits the
// reference itself):
//   * Microenvironment::agent_container is never initialised by the reference
//     (BioFVM_microenvironment.h:108) yet Basic_Agent::assign_position calls
//     through it (BioFVM_basic_agent.cpp:79): the harness installs a real
//     Agent_Container.
//   * agents are given positions inside the bounding box; otherwise
//     assign_position leaves current_voxel_index uninitialised
//     (BioFVM_basic_agent.cpp:69-73).  Out-of-box agents are rejected here.
//   * the cell step of the reference is an OpenMP loop that races when two
//     agents share a voxel (BioFVM_microenvironment.cpp:615-624); in parity
//     mode the harness runs that one call with a single OpenMP thread so the
//     agent order is the sequential order.
//   * bulk supply/target/uptake callbacks (BioFVM_microenvironment.h:130-132)
//     are installed as functions that read per-voxel tables set by the caller.

#include "BioFVM.h"

#include <omp.h>
#include <chrono>
#include <cstring>
#include <vector>

using namespace BioFVM;

namespace {

struct RefHarness {
  Microenvironment* M = nullptr;
  std::vector<Basic_Agent*> agents;
  std::vector<double> supply, target, uptake;  // [N][S] tables for callbacks
  int threads = 1;
  int cells_single_thread = 1;
};

RefHarness* g_active = nullptr;  // callbacks have no user pointer

void supply_cb(Microenvironment*, int n, std::vector<double>* dst) {
  const size_t S = dst->size();
  for (size_t s = 0; s < S; ++s) (*dst)[s] = g_active->supply[n * S + s];
}
void target_cb(Microenvironment*, int n, std::vector<double>* dst) {
  const size_t S = dst->size();
  for (size_t s = 0; s < S; ++s) (*dst)[s] = g_active->target[n * S + s];
}
void uptake_cb(Microenvironment*, int n, std::vector<double>* dst) {
  const size_t S = dst->size();
  for (size_t s = 0; s < S; ++s) (*dst)[s] = g_active->uptake[n * S + s];
}

}  // namespace

extern "C" {

void* refh_create(int num_densities) {
  RefHarness* h = new RefHarness;
  h->M = new Microenvironment();
  h->M->agent_container = new Agent_Container();
  // Microenvironment() starts with one density; grow to the requested count
  // through the reference's own add_density (BioFVM_microenvironment.cpp:325).
  for (int s = 1; s < num_densities; ++s) h->M->add_density();
  h->M->diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
  g_active = h;
  return h;
}

void refh_destroy(void* hp) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  // Agents are owned by the reference's global registry; remove ours from it.
  for (Basic_Agent* a : h->agents) {
    for (size_t i = 0; i < all_basic_agents.size(); ++i)
      if (all_basic_agents[i] == a) {
        all_basic_agents[i] = all_basic_agents.back();
        all_basic_agents.pop_back();
        break;
      }
    delete a;
  }
  if (g_active == h) g_active = nullptr;
  // The reference keeps a global default-microenvironment pointer (the first
  // Microenvironment ever built) that every new Basic_Agent registers with
  // first (BioFVM_basic_agent.cpp:51-53); that one object is kept alive.
  if (h->M != get_default_microenvironment()) {
    delete h->M->agent_container;
    delete h->M;
  }
  delete h;
}

void refh_set_threads(void* hp, int threads, int cells_single_thread) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  h->threads = threads > 0 ? threads : omp_get_num_procs();
  h->cells_single_thread = cells_single_thread;
  omp_set_num_threads(h->threads);
}

void refh_resize_space(void* hp, double x0, double x1, double y0, double y1, double z0,
                       double z1, double dx, double dy, double dz) {
  static_cast<RefHarness*>(hp)->M->resize_space(x0, x1, y0, y1, z0, z1, dx, dy, dz);
}

void refh_resize_space_nodes(void* hp, double x0, double x1, double y0, double y1,
                             double z0, double z1, int nx, int ny, int nz) {
  static_cast<RefHarness*>(hp)->M->resize_space(x0, x1, y0, y1, z0, z1, nx, ny, nz);
}

void refh_mesh_info(void* hp, int* nxyz, double* geom) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  nxyz[0] = (int)M->mesh.x_coordinates.size();
  nxyz[1] = (int)M->mesh.y_coordinates.size();
  nxyz[2] = (int)M->mesh.z_coordinates.size();
  nxyz[3] = M->number_of_densities();
  nxyz[4] = M->mesh.uniform_mesh ? 1 : 0;
  geom[0] = M->mesh.dx;
  geom[1] = M->mesh.dy;
  geom[2] = M->mesh.dz;
  geom[3] = M->mesh.dV;
  for (int i = 0; i < 6; ++i) geom[4 + i] = M->mesh.bounding_box[i];
}

void refh_set_coefficients(void* hp, const double* D, const double* decay) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  for (int s = 0; s < M->number_of_densities(); ++s) {
    M->diffusion_coefficients[s] = D[s];
    M->decay_rates[s] = decay[s];
  }
}

void refh_set_densities(void* hp, const double* p) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  const int S = M->number_of_densities();
  for (int n = 0; n < M->number_of_voxels(); ++n) {
    std::vector<double>& v = M->density_vector(n);
    for (int s = 0; s < S; ++s) v[s] = p[(size_t)n * S + s];
  }
}

void refh_get_densities(void* hp, double* p) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  const int S = M->number_of_densities();
  for (int n = 0; n < M->number_of_voxels(); ++n) {
    const std::vector<double>& v = M->density_vector(n);
    for (int s = 0; s < S; ++s) p[(size_t)n * S + s] = v[s];
  }
}

// Installs the three bulk callbacks.  NULL tables keep the reference default
// (zero_function, BioFVM_microenvironment.cpp:62-67,118-120).
void refh_set_bulk(void* hp, const double* supply, const double* target,
                   const double* uptake) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  const size_t NS = (size_t)h->M->number_of_voxels() * h->M->number_of_densities();
  if (supply) {
    h->supply.assign(supply, supply + NS);
    h->M->bulk_supply_rate_function = supply_cb;
  }
  if (target) {
    h->target.assign(target, target + NS);
    h->M->bulk_supply_target_densities_function = target_cb;
  }
  if (uptake) {
    h->uptake.assign(uptake, uptake + NS);
    h->M->bulk_uptake_rate_function = uptake_cb;
  }
  g_active = h;
}

void refh_add_dirichlet(void* hp, int voxel, const double* value) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  std::vector<double> v(value, value + M->number_of_densities());
  M->add_dirichlet_node(voxel, v);
}

void refh_update_dirichlet(void* hp, int voxel, const double* value) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  std::vector<double> v(value, value + M->number_of_densities());
  M->update_dirichlet_node(voxel, v);
}

// Creates one agent the way the reference drivers do
// (examples/performance_test_numcells.cpp:150-155): create_basic_agent,
// register_microenvironment, assign_position, volume, rates, then
// set_internal_uptake_constants(dt).  Returns the agent's voxel or -1 when
// the position is outside the box.
int refh_add_agent(void* hp, double x, double y, double z, double volume,
                   const double* secretion, const double* saturation,
                   const double* uptake, double dt) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  Microenvironment* M = h->M;
  if (!M->mesh.is_position_valid(x, y, z)) return -1;
  Basic_Agent* a = create_basic_agent();
  a->register_microenvironment(M);
  a->assign_position(x, y, z);
  a->volume = volume;
  const int S = M->number_of_densities();
  for (int s = 0; s < S; ++s) {
    (*a->secretion_rates)[s] = secretion[s];
    (*a->saturation_densities)[s] = saturation[s];
    (*a->uptake_rates)[s] = uptake[s];
  }
  a->set_internal_uptake_constants(dt);
  h->agents.push_back(a);
  return a->nearest_voxel_index();
}

// 3 = diffusion_decay_solver__constant_coefficients_LOD_3D (the default),
// 2 = diffusion_decay_solver__constant_coefficients_LOD_2D.
void refh_set_solver(void* hp, int dims) {
  static_cast<RefHarness*>(hp)->M->diffusion_decay_solver =
      dims == 2 ? diffusion_decay_solver__constant_coefficients_LOD_2D
                : diffusion_decay_solver__constant_coefficients_LOD_3D;
}

void refh_step_bulk(void* hp, double dt) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  g_active = h;
  h->M->simulate_bulk_sources_and_sinks(dt);
}

void refh_step_cells(void* hp, double dt) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  if (h->cells_single_thread) omp_set_num_threads(1);
  h->M->simulate_cell_sources_and_sinks(h->agents, dt);
  if (h->cells_single_thread) omp_set_num_threads(h->threads);
}

void refh_step_diffusion(void* hp, double dt) {
  static_cast<RefHarness*>(hp)->M->simulate_diffusion_decay(dt);
}

void refh_apply_dirichlet(void* hp) { static_cast<RefHarness*>(hp)->M->apply_dirichlet_conditions(); }

// One full step in the canonical order bulk -> cells -> diffusion
// (examples/performance_test_numcells.cpp:177-179).  flags bit0 = bulk,
// bit1 = cells, bit2 = diffusion.  Returns wall seconds of the loop
// (steady_clock), the reference's own TIC/TOC use clock() CPU time.
double refh_run(void* hp, double dt, int nsteps, int flags) {
  RefHarness* h = static_cast<RefHarness*>(hp);
  g_active = h;
  auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < nsteps; ++it) {
    if (flags & 1) h->M->simulate_bulk_sources_and_sinks(dt);
    if (flags & 2) refh_step_cells(hp, dt);
    if (flags & 4) h->M->simulate_diffusion_decay(dt);
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

int refh_num_threads(void) { return omp_get_max_threads(); }

// Microenvironment::compute_all_gradient_vectors (BioFVM_microenvironment.cpp:
// 702-787), then every voxel's gradient_vector(n) as [N][S][3].  The
// reference reads its jumps from the LOD_3D setup (BioFVM_solvers.cpp:
// 101-103): run a diffusion step first.
void refh_gradients(void* hp, double* out) {
  Microenvironment* M = static_cast<RefHarness*>(hp)->M;
  M->compute_all_gradient_vectors();
  const int S = M->number_of_densities();
  for (int n = 0; n < M->number_of_voxels(); ++n) {
    std::vector<gradient>& g = M->gradient_vector(n);
    for (int s = 0; s < S; ++s)
      for (int c = 0; c < 3; ++c) out[((size_t)n * S + s) * 3 + c] = g[s][c];
  }
}

}  // extern "C"
