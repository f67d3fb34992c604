// Microenvironment with BioFVM's public API (BioFVM_microenvironment.h:45-253)
// whose transport path runs on one GPU through libbfvm.so.
//
// The density field lives on the device.  density_vector() / operator() /
// nearest_density_vector() hand out references into a host mirror that is
// refreshed from the device on first access after a step, and that is sent
// back before the next simulate_* call (the mirror is assumed modified once a
// reference has been handed out).  Bulk supply/target/uptake callbacks run on
// the host for every voxel at every simulate_bulk_sources_and_sinks, into
// per-voxel vectors that persist between steps and are modified in place
// exactly as the reference modifies its own (:595-610); the voxels whose
// update is not the identity go to the device.
#ifndef __BioFVM_microenvironment_h__
#define __BioFVM_microenvironment_h__

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "BioFVM_agent_container.h"
#include "BioFVM_mesh.h"

struct bfvm_solver;

namespace BioFVM {

typedef std::vector<double> gradient;

class Basic_Agent;

class Microenvironment {
 private:
  friend void diffusion_decay_solver__constant_coefficients_LOD_3D(Microenvironment& S, double dt);
  friend void diffusion_decay_solver__constant_coefficients_LOD_2D(Microenvironment& S, double dt);
  friend class Basic_Agent;

  bfvm_solver* solver_;
  // host mirror of the device field, [voxel][substrate]
  std::vector<std::vector<double> > host_;
  std::atomic<bool> host_valid_;   // mirror holds the device values
  std::atomic<bool> host_dirty_;   // mirror may be newer than the device
  std::mutex mirror_mutex_;
  // coefficient and bulk-rate state last sent to the device
  std::vector<double> sent_D_, sent_decay_;
  bool rates_dirty_;
  // the reference's bulk_source_sink_solver_temp1/2/3: per-voxel vectors
  // handed to the callbacks and modified in place after them
  std::vector<std::vector<double> > bulk_temp1_, bulk_temp2_, bulk_temp3_;
  std::vector<int64_t> sent_bulk_vox_;
  std::vector<double> sent_bulk_rates_;
  uint64_t sent_agent_epoch_;
  const void* sent_agent_list_;
  std::vector<int> dirichlet_indices;
  std::vector<std::vector<double> > dirichlet_value_vectors;
  // gradient vectors [voxel][substrate][3] (BioFVM_microenvironment.h:65-66)
  std::vector<std::vector<gradient> > gradient_vectors;
  std::vector<bool> gradient_vector_computed;
  void size_gradient_vectors();

  void ensure_solver();
  void copy_state(const Microenvironment& o);
  void sync_to_host();
  void sync_to_device();
  void prepare_step(bool bulk, bool cells, std::vector<Basic_Agent*>* list, double dt = 0.0);
  void upload_agents(std::vector<Basic_Agent*>& list);
  void upload_bulk_rates(double dt);
  void after_resize();
  std::vector<double>& mirror(int n);

 public:
  Cartesian_Mesh mesh;
  Agent_Container* agent_container;
  std::string spatial_units;
  std::string time_units;
  std::string name;

  std::vector<std::string> density_names;
  std::vector<std::string> density_units;

  std::vector<double> diffusion_coefficients;
  std::vector<double> decay_rates;

  std::vector<std::vector<double> > supply_target_densities_times_supply_rates;
  std::vector<std::vector<double> > supply_rates;
  std::vector<std::vector<double> > uptake_rates;
  void update_rates(void);

  Microenvironment();
  Microenvironment(std::string name);
  ~Microenvironment();
  // A copy holds the state and a host snapshot of the densities; it gets its
  // own device solver only if a step is run on it (drivers pass
  // Microenvironments by value to their output routines).
  Microenvironment(const Microenvironment& other);
  Microenvironment& operator=(const Microenvironment& other);

  void (*diffusion_decay_solver)(Microenvironment&, double);
  void (*bulk_supply_rate_function)(Microenvironment* pMicroenvironment, int voxel_index,
                                    std::vector<double>* write_destination);
  void (*bulk_supply_target_densities_function)(Microenvironment* pMicroenvironment,
                                                int voxel_index,
                                                std::vector<double>* write_destination);
  void (*bulk_uptake_rate_function)(Microenvironment* pMicroenvironment, int voxel_index,
                                    std::vector<double>* write_destination);

  int number_of_densities(void);
  int number_of_voxels(void);
  int number_of_voxel_faces(void);

  void auto_choose_diffusion_decay_solver(void);

  void resize_space(int x_nodes, int y_nodes, int z_nodes);
  void resize_space(double x_start, double x_end, double y_start, double y_end, double z_start,
                    double z_end, int x_nodes, int y_nodes, int z_nodes);
  void resize_space(double x_start, double x_end, double y_start, double y_end, double z_start,
                    double z_end, double dx_new, double dy_new, double dz_new);
  void resize_space_uniform(double x_start, double x_end, double y_start, double y_end,
                            double z_start, double z_end, double dx_new);

  void resize_densities(int new_size);
  void add_density(void);
  void add_density(std::string name, std::string units);
  void add_density(std::string name, std::string units, double diffusion_constant,
                   double decay_rate);

  void set_density(int index, std::string name, std::string units);
  void set_density(int index, std::string name, std::string units, double diffusion_constant,
                   double decay_rate);

  int voxel_index(int i, int j, int k);
  std::vector<int> cartesian_indices(int n);

  int nearest_voxel_index(std::vector<double>& position);
  std::vector<int> nearest_cartesian_indices(std::vector<double>& position);
  Voxel& nearest_voxel(std::vector<double>& position);
  Voxel& voxels(int voxel_index);
  std::vector<double>& nearest_density_vector(std::vector<double>& position);
  std::vector<double>& nearest_density_vector(int voxel_index);

  std::vector<double>& operator()(int i, int j, int k);
  std::vector<double>& operator()(int i, int j);
  std::vector<double>& operator()(int n);

  // gradients (BioFVM_microenvironment.h:176-184)
  std::vector<gradient>& gradient_vector(int i, int j, int k);
  std::vector<gradient>& gradient_vector(int i, int j);
  std::vector<gradient>& gradient_vector(int n);
  std::vector<gradient>& nearest_gradient_vector(std::vector<double>& position);
  void compute_all_gradient_vectors(void);
  void compute_gradient_vector(int n);
  void reset_all_gradient_vectors(void);

  std::vector<double>& density_vector(int i, int j, int k);
  std::vector<double>& density_vector(int i, int j);
  std::vector<double>& density_vector(int n);

  void simulate_diffusion_decay(double dt);
  void simulate_bulk_sources_and_sinks(double dt);
  void simulate_cell_sources_and_sinks(std::vector<Basic_Agent*>& basic_agent_list, double dt);
  void simulate_cell_sources_and_sinks(double dt);

  void display_information(std::ostream& os);

  void add_dirichlet_node(int voxel_index, std::vector<double>& value);
  void update_dirichlet_node(int voxel_index, std::vector<double>& new_value);
  void remove_dirichlet_node(int voxel_index);
  void apply_dirichlet_conditions(void);

  void write_to_matlab(std::string filename);

  // ---- beyond the reference API -------------------------------------------
  // The whole step bulk -> cells -> diffusion in one call (fused kernels).
  void simulate_step(double dt, bool bulk = true, bool cells = true);
  // Recompute the Thomas coefficients at the next diffusion step (the
  // reference computes them once and never again).
  void reset_diffusion_solver(void);
  // The underlying C-ABI handle (created on first use for a copy).
  bfvm_solver* device_solver(void) {
    ensure_solver();
    return solver_;
  }
};

void zero_function(std::vector<double>& position, std::vector<double>& input,
                   std::vector<double>* destination);
void one_function(std::vector<double>& position, std::vector<double>& input,
                  std::vector<double>* destination);
void zero_function(Microenvironment* pMicroenvironment, int voxel_index,
                   std::vector<double>* write_destination);
void one_function(Microenvironment* pMicroenvironment, int voxel_index,
                  std::vector<double>* write_destination);

Microenvironment* get_default_microenvironment(void);
void set_default_microenvironment(Microenvironment* M);

}  // namespace BioFVM

#endif
