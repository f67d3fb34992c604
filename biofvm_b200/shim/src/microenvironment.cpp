// Microenvironment of the drop-in headers over libbfvm.so (include/bfvm.h).
// Reference behaviour cited per function (BioFVM_microenvironment.cpp).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "BioFVM.h"
#include "bfvm.h"

namespace BioFVM {

namespace {

Microenvironment* g_default = nullptr;

void check(int rc, const char* what) {
  if (rc != BFVM_OK)
    throw std::runtime_error(std::string(what) + ": " + bfvm_last_error());
}

int device_index() {
  const char* d = std::getenv("BFVM_DEVICE");
  return d ? std::atoi(d) : 0;
}

}  // namespace

Microenvironment* get_default_microenvironment(void) { return g_default; }
void set_default_microenvironment(Microenvironment* M) { g_default = M; }

// BioFVM_microenvironment.cpp:48-74
void zero_function(std::vector<double>&, std::vector<double>&, std::vector<double>* dst) {
  for (double& x : *dst) x = 0.0;
}
void one_function(std::vector<double>&, std::vector<double>&, std::vector<double>* dst) {
  for (double& x : *dst) x = 1.0;
}
void zero_function(Microenvironment*, int, std::vector<double>* dst) {
  for (double& x : *dst) x = 0.0;
}
void one_function(Microenvironment*, int, std::vector<double>* dst) {
  for (double& x : *dst) x = 1.0;
}

// BioFVM_microenvironment.cpp:88-139: one voxel, one density, LOD_3D solver
Microenvironment::Microenvironment()
    : solver_(nullptr),
      host_valid_(false),
      host_dirty_(false),
      rates_dirty_(true),
      sent_agent_epoch_(~0ull),
      sent_agent_list_(nullptr) {
  check(bfvm_create(&solver_, device_index()), "bfvm_create");
  name = "unnamed";
  spatial_units = "none";
  time_units = "none";
  mesh.resize(1, 1, 1);
  agent_container = new Agent_Container;
  density_names.assign(1, "unnamed");
  density_units.assign(1, "none");
  diffusion_coefficients.assign(1, 0.0);
  decay_rates.assign(1, 0.0);
  diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
  bulk_supply_rate_function = zero_function;
  bulk_supply_target_densities_function = zero_function;
  bulk_uptake_rate_function = zero_function;
  if (g_default == nullptr) g_default = this;
}

// The reference's Microenvironment(std::string) builds a temporary and leaves
// *this uninitialised (BioFVM_microenvironment.cpp:141-145); here it builds
// this object and names it.
Microenvironment::Microenvironment(std::string nm) : Microenvironment() { name = nm; }

Microenvironment::~Microenvironment() {
  if (g_default == this) g_default = nullptr;
  delete agent_container;
  if (solver_) bfvm_destroy(solver_);
}

void Microenvironment::copy_state(const Microenvironment& o) {
  Microenvironment& src = const_cast<Microenvironment&>(o);
  mesh = o.mesh;
  spatial_units = o.spatial_units;
  time_units = o.time_units;
  name = o.name;
  density_names = o.density_names;
  density_units = o.density_units;
  diffusion_coefficients = o.diffusion_coefficients;
  decay_rates = o.decay_rates;
  supply_target_densities_times_supply_rates = o.supply_target_densities_times_supply_rates;
  supply_rates = o.supply_rates;
  uptake_rates = o.uptake_rates;
  diffusion_decay_solver = o.diffusion_decay_solver;
  bulk_supply_rate_function = o.bulk_supply_rate_function;
  bulk_supply_target_densities_function = o.bulk_supply_target_densities_function;
  bulk_uptake_rate_function = o.bulk_uptake_rate_function;
  dirichlet_indices = o.dirichlet_indices;
  dirichlet_value_vectors = o.dirichlet_value_vectors;
  // host snapshot of the source's densities
  if (!src.host_valid_.load() && src.solver_) {
    std::lock_guard<std::mutex> g(src.mirror_mutex_);
    if (!src.host_valid_.load()) {
      src.sync_to_host();
      src.host_valid_.store(true);
    }
  }
  host_ = src.host_;
  if (host_.size() != mesh.voxels.size())
    host_.assign(mesh.voxels.size(), std::vector<double>(density_names.size(), 0.0));
  host_valid_.store(true);
  host_dirty_.store(true);  // the device copy, when made, starts from it
  rates_dirty_ = true;
  sent_D_.clear();
  sent_decay_.clear();
  sent_agent_epoch_ = ~0ull;
  sent_agent_list_ = nullptr;
  bulk_temp1_ = o.bulk_temp1_;
  bulk_temp2_ = o.bulk_temp2_;
  bulk_temp3_ = o.bulk_temp3_;
  sent_bulk_vox_.clear();
  sent_bulk_rates_.clear();
}

Microenvironment::Microenvironment(const Microenvironment& o)
    : solver_(nullptr), host_valid_(false), host_dirty_(false), rates_dirty_(true) {
  agent_container = new Agent_Container;
  copy_state(o);
}

Microenvironment& Microenvironment::operator=(const Microenvironment& o) {
  if (this == &o) return *this;
  if (solver_) bfvm_destroy(solver_);
  solver_ = nullptr;
  copy_state(o);
  return *this;
}

// Gives a copy its device solver: the mesh exactly, the densities, the
// Dirichlet nodes; coefficients, rates and agents follow in prepare_step.
void Microenvironment::ensure_solver() {
  if (solver_) return;
  check(bfvm_create(&solver_, device_index()), "bfvm_create");
  const int nxyz[3] = {(int)mesh.x_coordinates.size(), (int)mesh.y_coordinates.size(),
                       (int)mesh.z_coordinates.size()};
  const double geom[10] = {mesh.dx, mesh.dy, mesh.dz, mesh.dV, mesh.bounding_box[0],
                           mesh.bounding_box[1], mesh.bounding_box[2], mesh.bounding_box[3],
                           mesh.bounding_box[4], mesh.bounding_box[5]};
  check(bfvm_resize_densities(solver_, number_of_densities()), "bfvm_resize_densities");
  check(bfvm_set_mesh(solver_, nxyz, geom, mesh.uniform_mesh ? 1 : 0), "bfvm_set_mesh");
  for (size_t d = 0; d < dirichlet_indices.size(); ++d)
    check(bfvm_add_dirichlet_node(solver_, dirichlet_indices[d], dirichlet_value_vectors[d].data()),
          "bfvm_add_dirichlet_node");
  host_dirty_.store(true);
}

// ---- host mirror ------------------------------------------------------------

void Microenvironment::sync_to_host() {
  ensure_solver();
  const int S = number_of_densities();
  const size_t N = mesh.voxels.size();
  std::vector<double> flat(N * S);
  check(bfvm_get_densities(solver_, flat.data()), "bfvm_get_densities");
  if (host_.size() != N) host_.assign(N, std::vector<double>(S));
  for (size_t n = 0; n < N; ++n) host_[n].assign(flat.begin() + n * S, flat.begin() + (n + 1) * S);
}

void Microenvironment::sync_to_device() {
  ensure_solver();
  if (!host_dirty_.load()) return;
  const int S = number_of_densities();
  const size_t N = mesh.voxels.size();
  std::vector<double> flat(N * S);
  for (size_t n = 0; n < N; ++n) std::copy_n(host_[n].data(), S, &flat[n * S]);
  check(bfvm_set_densities(solver_, flat.data()), "bfvm_set_densities");
  host_dirty_.store(false);
}

std::vector<double>& Microenvironment::mirror(int n) {
  if (!host_valid_.load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> g(mirror_mutex_);
    if (!host_valid_.load(std::memory_order_relaxed)) {
      sync_to_host();
      host_valid_.store(true, std::memory_order_release);
    }
  }
  host_dirty_.store(true, std::memory_order_relaxed);
  return host_[n];
}

void Microenvironment::after_resize() {
  host_.clear();
  host_valid_.store(false);
  host_dirty_.store(false);
  rates_dirty_ = true;
  sent_agent_epoch_ = ~0ull;
  sent_D_.clear();
  sent_decay_.clear();
  dirichlet_indices.clear();
  dirichlet_value_vectors.clear();
  bulk_temp1_.clear();
  bulk_temp2_.clear();
  bulk_temp3_.clear();
  sent_bulk_vox_.clear();
  sent_bulk_rates_.clear();
}

// ---- before every device step ---------------------------------------------

void Microenvironment::upload_bulk_rates(double dt) {
  // simulate_bulk_sources_and_sinks (BioFVM_microenvironment.cpp:584-613):
  // the three callbacks (BioFVM_microenvironment.h:130-132) write into
  // per-voxel vectors allocated once with zeros (:586-593).  After the
  // update the reference leaves temp2 = S*T and temp3 = 1 + dt*(U+S) in those
  // vectors (:603-607), so a callback that skips a voxel finds these values
  // there at the next step; the same vectors and the same in-place
  // operations are kept here.  The device receives (S, T, U) as the
  // callbacks left them for every voxel whose update is not the identity.
  const int S = number_of_densities();
  const int N = number_of_voxels();
  if ((int)bulk_temp1_.size() != N) {
    const std::vector<double> zero(S, 0.0);
    bulk_temp1_.assign(N, zero);
    bulk_temp2_.assign(N, zero);
    bulk_temp3_.assign(N, zero);
  }
  std::vector<char> keep(N, 0);
  std::vector<double> rates((size_t)N * 3 * S);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    std::vector<double>& t1 = bulk_temp1_[n];
    std::vector<double>& t2 = bulk_temp2_[n];
    std::vector<double>& t3 = bulk_temp3_[n];
    bulk_supply_rate_function(this, n, &t1);
    bulk_supply_target_densities_function(this, n, &t2);
    bulk_uptake_rate_function(this, n, &t3);
    bool identity = true;
    double* r = &rates[(size_t)n * 3 * S];
    for (int s = 0; s < S; ++s) {
      const double sv = t1[s], tv = t2[s], uv = t3[s];
      identity = identity && tv * sv == 0.0 && uv + sv == 0.0;
      r[s] = sv;
      r[S + s] = tv;
      r[2 * S + s] = uv;
    }
    keep[n] = !identity;
    // the reference's in-place updates of its temporaries (:602-607)
    for (int s = 0; s < S; ++s) {
      t2[s] *= t1[s];
      t3[s] += t1[s];
      t3[s] *= dt;
      t3[s] += 1.0;
    }
  }
  std::vector<int64_t> vox;
  for (int n = 0; n < N; ++n)
    if (keep[n]) vox.push_back(n);
  const size_t E = vox.size();
  std::vector<double> sup(E * S), tar(E * S), upt(E * S), packed;
  for (size_t e = 0; e < E; ++e) {
    const double* r = &rates[(size_t)vox[e] * 3 * S];
    std::copy_n(r, S, &sup[e * S]);
    std::copy_n(r + S, S, &tar[e * S]);
    std::copy_n(r + 2 * S, S, &upt[e * S]);
  }
  packed.reserve(3 * E * S);
  packed.insert(packed.end(), sup.begin(), sup.end());
  packed.insert(packed.end(), tar.begin(), tar.end());
  packed.insert(packed.end(), upt.begin(), upt.end());
  if (vox == sent_bulk_vox_ && packed == sent_bulk_rates_ && !rates_dirty_) return;
  check(bfvm_set_bulk_rates_sparse(solver_, (int64_t)E, vox.data(), sup.data(), tar.data(),
                                   upt.data()),
        "bfvm_set_bulk_rates_sparse");
  sent_bulk_vox_.swap(vox);
  sent_bulk_rates_.swap(packed);
  rates_dirty_ = false;
}

void Microenvironment::upload_agents(std::vector<Basic_Agent*>& list) {
  const int S = number_of_densities();
  const size_t A = list.size();
  std::vector<int64_t> vox(A);
  std::vector<double> t1(A * S), t2(A * S);
  for (size_t a = 0; a < A; ++a) {
    Basic_Agent* p = list[a];
    vox[a] = p->current_voxel_index;
    for (int s = 0; s < S; ++s) {
      t1[a * S + s] = s < (int)p->cell_source_sink_solver_temp1.size()
                          ? p->cell_source_sink_solver_temp1[s] : 0.0;
      t2[a * S + s] = s < (int)p->cell_source_sink_solver_temp2.size()
                          ? p->cell_source_sink_solver_temp2[s] : 1.0;
    }
  }
  check(bfvm_set_agents(solver_, (int64_t)A, vox.data(), t1.data(), t2.data()),
        "bfvm_set_agents");
  sent_agent_epoch_ = basic_agent_epoch();
  sent_agent_list_ = &list;
}

void Microenvironment::prepare_step(bool bulk, bool cells, std::vector<Basic_Agent*>* list,
                                    double dt) {
  sync_to_device();
  if (sent_D_ != diffusion_coefficients || sent_decay_ != decay_rates) {
    for (int s = 0; s < number_of_densities(); ++s)
      check(bfvm_set_density_coefficients(solver_, s, diffusion_coefficients[s], decay_rates[s]),
            "bfvm_set_density_coefficients");
    sent_D_ = diffusion_coefficients;
    sent_decay_ = decay_rates;
  }
  if (bulk) upload_bulk_rates(dt);
  if (cells) {
    std::vector<Basic_Agent*>& l = list ? *list : all_basic_agents;
    if (sent_agent_epoch_ != basic_agent_epoch() || sent_agent_list_ != &l) upload_agents(l);
  }
}

// ---- sizes, densities, geometry -------------------------------------------

int Microenvironment::number_of_densities(void) { return (int)density_names.size(); }
int Microenvironment::number_of_voxels(void) { return (int)mesh.voxels.size(); }
int Microenvironment::number_of_voxel_faces(void) { return 0; }

void Microenvironment::auto_choose_diffusion_decay_solver(void) {
  // BioFVM_microenvironment.cpp:515-526 selects the (no-op) explicit solver
  diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_explicit;
  std::cout << "Warning: auto-selection of diffusion-decay-source/sink solver not fully "
               "implemented!"
            << std::endl;
}

void Microenvironment::resize_space(int nx, int ny, int nz) {
  ensure_solver();
  mesh.resize(nx, ny, nz);
  check(bfvm_resize_space_nodes(solver_, -0.5, nx - 1 + .5, -0.5, ny - 1 + .5, -0.5,
                                nz - 1 + .5, nx, ny, nz),
        "bfvm_resize_space_nodes");
  after_resize();
}

void Microenvironment::resize_space(double x0, double x1, double y0, double y1, double z0,
                                    double z1, int nx, int ny, int nz) {
  ensure_solver();
  mesh.resize(x0, x1, y0, y1, z0, z1, nx, ny, nz);
  check(bfvm_resize_space_nodes(solver_, x0, x1, y0, y1, z0, z1, nx, ny, nz),
        "bfvm_resize_space_nodes");
  after_resize();
}

void Microenvironment::resize_space(double x0, double x1, double y0, double y1, double z0,
                                    double z1, double dx, double dy, double dz) {
  ensure_solver();
  mesh.resize(x0, x1, y0, y1, z0, z1, dx, dy, dz);
  check(bfvm_resize_space(solver_, x0, x1, y0, y1, z0, z1, dx, dy, dz), "bfvm_resize_space");
  after_resize();
}

void Microenvironment::resize_space_uniform(double x0, double x1, double y0, double y1,
                                            double z0, double z1, double dx) {
  resize_space(x0, x1, y0, y1, z0, z1, dx, dx, dx);
}

void Microenvironment::resize_densities(int new_size) {
  // BioFVM_microenvironment.cpp:292-323: all densities zero, coefficients 0
  ensure_solver();
  check(bfvm_resize_densities(solver_, new_size), "bfvm_resize_densities");
  density_names.assign(new_size, "unnamed");
  density_units.assign(new_size, "none");
  diffusion_coefficients.assign(new_size, 0.0);
  decay_rates.assign(new_size, 0.0);
  after_resize();
}

void Microenvironment::add_density(std::string nm, std::string units, double D, double decay) {
  // BioFVM_microenvironment.cpp:404-441: one more density, zero everywhere
  sync_to_device();
  check(bfvm_add_density(solver_, D, decay), "bfvm_add_density");
  density_names.push_back(nm);
  density_units.push_back(units);
  diffusion_coefficients.push_back(D);
  decay_rates.push_back(decay);
  host_valid_.store(false);
  for (auto& v : dirichlet_value_vectors) v.push_back(0.0);
  rates_dirty_ = true;
  sent_agent_epoch_ = ~0ull;
}
void Microenvironment::add_density(void) { add_density("unnamed", "none", 0.0, 0.0); }
void Microenvironment::add_density(std::string nm, std::string units) {
  add_density(nm, units, 0.0, 0.0);
}

void Microenvironment::set_density(int index, std::string nm, std::string units) {
  density_names[index] = nm;
  density_units[index] = units;
}
void Microenvironment::set_density(int index, std::string nm, std::string units, double D,
                                   double decay) {
  density_names[index] = nm;
  density_units[index] = units;
  diffusion_coefficients[index] = D;
  decay_rates[index] = decay;
}

int Microenvironment::voxel_index(int i, int j, int k) { return mesh.voxel_index(i, j, k); }
std::vector<int> Microenvironment::cartesian_indices(int n) { return mesh.cartesian_indices(n); }
int Microenvironment::nearest_voxel_index(std::vector<double>& position) {
  return mesh.nearest_voxel_index(position);
}
std::vector<int> Microenvironment::nearest_cartesian_indices(std::vector<double>& position) {
  return mesh.nearest_cartesian_indices(position);
}
Voxel& Microenvironment::nearest_voxel(std::vector<double>& position) {
  return mesh.nearest_voxel(position);
}
Voxel& Microenvironment::voxels(int n) { return mesh.voxels[n]; }

std::vector<double>& Microenvironment::nearest_density_vector(std::vector<double>& position) {
  return mirror(mesh.nearest_voxel_index(position));
}
std::vector<double>& Microenvironment::nearest_density_vector(int n) { return mirror(n); }
std::vector<double>& Microenvironment::operator()(int i, int j, int k) {
  return mirror(voxel_index(i, j, k));
}
std::vector<double>& Microenvironment::operator()(int i, int j) {
  return mirror(voxel_index(i, j, 0));
}
std::vector<double>& Microenvironment::operator()(int n) { return mirror(n); }
std::vector<double>& Microenvironment::density_vector(int i, int j, int k) {
  return mirror(voxel_index(i, j, k));
}
std::vector<double>& Microenvironment::density_vector(int i, int j) {
  return mirror(voxel_index(i, j, 0));
}
std::vector<double>& Microenvironment::density_vector(int n) { return mirror(n); }

// ---- the step ----------------------------------------------------------------

void Microenvironment::simulate_diffusion_decay(double dt) {
  // BioFVM_microenvironment.cpp:502-513
  if (diffusion_decay_solver) {
    diffusion_decay_solver(*this, dt);
  } else {
    std::cout << "Warning: diffusion-reaction-source/sink solver not set for Microenvironment "
                 "object at "
              << this << ". Nothing happened!" << std::endl;
    std::cout << "   Consider using Microenvironment::auto_choose_diffusion_decay_solver(void) "
                 "... "
              << std::endl
              << std::endl;
  }
}

void Microenvironment::simulate_bulk_sources_and_sinks(double dt) {
  prepare_step(true, false, nullptr, dt);
  check(bfvm_simulate_bulk_sources_and_sinks(solver_, dt), "bfvm_simulate_bulk_sources_and_sinks");
  host_valid_.store(false);
}

void Microenvironment::simulate_cell_sources_and_sinks(std::vector<Basic_Agent*>& list,
                                                        double dt) {
  prepare_step(false, true, &list);
  check(bfvm_simulate_cell_sources_and_sinks(solver_, dt), "bfvm_simulate_cell_sources_and_sinks");
  host_valid_.store(false);
}

void Microenvironment::simulate_cell_sources_and_sinks(double dt) {
  prepare_step(false, true, nullptr);
  check(bfvm_simulate_cell_sources_and_sinks(solver_, dt), "bfvm_simulate_cell_sources_and_sinks");
  host_valid_.store(false);
}

void Microenvironment::simulate_step(double dt, bool bulk, bool cells) {
  prepare_step(bulk, cells, nullptr, dt);
  const int flags = BFVM_STEP_DIFFUSION | (bulk ? BFVM_STEP_BULK : 0) | (cells ? BFVM_STEP_CELLS : 0);
  const int rc = bfvm_step(solver_, dt, 1, flags);
  if (rc == BFVM_ERR_MESH) {
    std::cout << bfvm_last_error() << std::endl << std::endl;
    return;
  }
  check(rc, "bfvm_step");
  host_valid_.store(false);
}

void Microenvironment::reset_diffusion_solver(void) {
  ensure_solver();
  check(bfvm_reset_diffusion_setup(solver_), "bfvm_reset_diffusion_setup");
}

void Microenvironment::update_rates(void) {
  // BioFVM_microenvironment.cpp:635-656, and re-send the rates to the device
  const int N = number_of_voxels();
  const std::vector<double> zero(number_of_densities(), 0.0);
  if ((int)supply_target_densities_times_supply_rates.size() != N)
    supply_target_densities_times_supply_rates.assign(N, zero);
  if ((int)supply_rates.size() != N) supply_rates.assign(N, zero);
  if ((int)uptake_rates.size() != N) uptake_rates.assign(N, zero);
  for (int i = 0; i < N; ++i) {
    bulk_uptake_rate_function(this, i, &uptake_rates[i]);
    bulk_supply_rate_function(this, i, &supply_rates[i]);
    bulk_supply_target_densities_function(this, i, &supply_target_densities_times_supply_rates[i]);
    supply_target_densities_times_supply_rates[i] *= supply_rates[i];
  }
  rates_dirty_ = true;
}

// ---- gradients (BioFVM_microenvironment.cpp:660-858) -------------------------

void Microenvironment::size_gradient_vectors() {
  // as the reference's resize_* (:213-222): existing entries keep their values
  const int N = number_of_voxels(), S = number_of_densities();
  gradient_vectors.resize(N);
  for (auto& v : gradient_vectors) {
    v.resize(S);
    for (auto& g : v) g.resize(3, 0.0);
  }
  gradient_vector_computed.resize(N, false);
}

void Microenvironment::compute_all_gradient_vectors(void) {
  // On the device (bfvm_compute_all_gradient_vectors); the components the
  // reference writes -- axes along which the voxel has both neighbours --
  // are copied into the host vectors, the others keep their values.
  size_gradient_vectors();
  sync_to_device();
  check(bfvm_compute_all_gradient_vectors(solver_), "bfvm_compute_all_gradient_vectors");
  const int N = number_of_voxels(), S = number_of_densities();
  std::vector<double> g((size_t)N * S * 3);
  check(bfvm_get_gradient_vectors(solver_, g.data()), "bfvm_get_gradient_vectors");
  const int nx = (int)mesh.x_coordinates.size(), ny = (int)mesh.y_coordinates.size(),
            nz = (int)mesh.z_coordinates.size();
  for (int n = 0; n < N; ++n) {
    const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
    const bool in[3] = {i > 0 && i < nx - 1, j > 0 && j < ny - 1, k > 0 && k < nz - 1};
    for (int s = 0; s < S; ++s)
      for (int c = 0; c < 3; ++c)
        if (in[c]) gradient_vectors[n][s][c] = g[((size_t)n * S + s) * 3 + c];
    if (in[0] || in[1] || in[2]) gradient_vector_computed[n] = true;
  }
}

void Microenvironment::compute_gradient_vector(int n) {
  // :790-843, from the host copy of the densities
  size_gradient_vectors();
  const int nx = (int)mesh.x_coordinates.size(), ny = (int)mesh.y_coordinates.size(),
            nz = (int)mesh.z_coordinates.size();
  const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
  const int jump[3] = {1, nx, nx * ny};
  const bool in[3] = {i > 0 && i < nx - 1, j > 0 && j < ny - 1, k > 0 && k < nz - 1};
  const double two_d[3] = {mesh.dx * 2.0, mesh.dy * 2.0, mesh.dz * 2.0};
  const int S = number_of_densities();
  for (int c = 0; c < 3; ++c) {
    if (!in[c]) continue;
    const std::vector<double>& up = mirror(n + jump[c]);
    const std::vector<double>& down = mirror(n - jump[c]);
    for (int s = 0; s < S; ++s) {
      double v = up[s];
      v -= down[s];
      v /= two_d[c];
      gradient_vectors[n][s][c] = v;
    }
    gradient_vector_computed[n] = true;
  }
}

void Microenvironment::reset_all_gradient_vectors(void) {
  size_gradient_vectors();
  gradient_vector_computed.assign(number_of_voxels(), false);
}

std::vector<gradient>& Microenvironment::gradient_vector(int n) {
  size_gradient_vectors();
  if (!gradient_vector_computed[n]) compute_gradient_vector(n);
  return gradient_vectors[n];
}

std::vector<gradient>& Microenvironment::gradient_vector(int i, int j, int k) {
  return gradient_vector(mesh.voxel_index(i, j, k));
}

std::vector<gradient>& Microenvironment::gradient_vector(int i, int j) {
  return gradient_vector(mesh.voxel_index(i, j, 0));
}

std::vector<gradient>& Microenvironment::nearest_gradient_vector(std::vector<double>& position) {
  return gradient_vector(mesh.nearest_voxel_index(position));
}

// ---- Dirichlet nodes (BioFVM_microenvironment.cpp:146-197) ----------------

void Microenvironment::add_dirichlet_node(int n, std::vector<double>& value) {
  ensure_solver();
  mesh.voxels[n].is_Dirichlet = true;
  dirichlet_indices.push_back(n);
  dirichlet_value_vectors.push_back(value);
  check(bfvm_add_dirichlet_node(solver_, n, value.data()), "bfvm_add_dirichlet_node");
}

void Microenvironment::update_dirichlet_node(int n, std::vector<double>& value) {
  ensure_solver();
  size_t d = 0;
  while (d < dirichlet_indices.size() && dirichlet_indices[d] != n) ++d;
  if (d == dirichlet_indices.size()) {
    std::cout << "BioFVM Warning: No Dirichlet condition previously specified at voxel " << n
              << "! Creating a new one now ... " << std::endl;
    add_dirichlet_node(n, value);
    return;
  }
  dirichlet_value_vectors[d] = value;
  check(bfvm_update_dirichlet_node(solver_, n, value.data()), "bfvm_update_dirichlet_node");
}

void Microenvironment::remove_dirichlet_node(int n) {
  // The reference pops the value list twice and never the index list
  // (:186-187); here both lists lose exactly the removed node.
  ensure_solver();
  mesh.voxels[n].is_Dirichlet = false;
  size_t d = 0;
  while (d < dirichlet_indices.size() && dirichlet_indices[d] != n) ++d;
  if (d == dirichlet_indices.size()) {
    std::cout << "BioFVM Warning: No Dirichlet condition previously specified at voxel " << n
              << "! Nothing to remove!" << std::endl;
    return;
  }
  dirichlet_indices[d] = dirichlet_indices.back();
  dirichlet_value_vectors[d] = dirichlet_value_vectors.back();
  dirichlet_indices.pop_back();
  dirichlet_value_vectors.pop_back();
  check(bfvm_remove_dirichlet_node(solver_, n), "bfvm_remove_dirichlet_node");
}

void Microenvironment::apply_dirichlet_conditions(void) {
  sync_to_device();
  check(bfvm_apply_dirichlet_conditions(solver_), "bfvm_apply_dirichlet_conditions");
  host_valid_.store(false);
}

// ---- output ----------------------------------------------------------------

void Microenvironment::display_information(std::ostream& os) {
  // BioFVM_microenvironment.cpp:528-546
  os << std::endl << "Microenvironment summary: " << name << ": " << std::endl;
  mesh.display_information(os);
  os << "Densities: (" << number_of_densities() << " total)" << std::endl;
  for (size_t i = 0; i < density_names.size(); ++i) {
    os << "   " << density_names[i] << ":" << std::endl
       << "     units: " << density_units[i] << std::endl
       << "     diffusion coefficient: " << diffusion_coefficients[i] << " " << spatial_units
       << "^2 / " << time_units << std::endl
       << "     decay rate: " << decay_rates[i] << " " << time_units << "^-1" << std::endl
       << "     diffusion length scale: "
       << std::sqrt(diffusion_coefficients[i] / (1e-12 + decay_rates[i])) << " "
       << spatial_units << std::endl
       << std::endl;
  }
  os << std::endl;
}

void Microenvironment::write_to_matlab(std::string filename) {
  // BioFVM_microenvironment.cpp:557-580: one column per voxel holding
  // x, y, z, volume, then the densities
  const int S = number_of_densities();
  const size_t N = mesh.voxels.size();
  std::vector<double> flat(N * S);
  if (host_valid_.load() && (host_dirty_.load() || solver_ == nullptr)) {
    for (size_t n = 0; n < N; ++n) std::copy_n(host_[n].data(), S, &flat[n * S]);
  } else {
    ensure_solver();
    check(bfvm_get_densities(solver_, flat.data()), "bfvm_get_densities");
  }
  FILE* fp = write_matlab_header(4 + S, (int)N, filename, "multiscale_microenvironment");
  if (!fp) return;
  std::vector<double> col(4 + S);
  for (size_t n = 0; n < N; ++n) {
    const Voxel& v = mesh.voxels[n];
    col[0] = v.center[0];
    col[1] = v.center[1];
    col[2] = v.center[2];
    col[3] = v.volume;
    std::copy_n(&flat[n * S], S, &col[4]);
    std::fwrite(col.data(), sizeof(double), col.size(), fp);
  }
  std::fclose(fp);
}

}  // namespace BioFVM
