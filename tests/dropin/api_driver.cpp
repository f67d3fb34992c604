// A driver of the BioFVM API for the drop-in test: built once against the
// reference sources and once against biofvm_b200's headers, it exercises
// what the reference's example programs leave out -- agents with secretion
// and uptake, Dirichlet nodes, direct density writes, the combined and the
// separate step calls, gradients (all voxels, and the lazy per-voxel path)
// -- and prints every number it reads, one per line, for the test to compare.
#include <cmath>
#include <cstdio>
#include <vector>

#include "BioFVM.h"
#include "BioFVM_agent_container.h"

using namespace BioFVM;

static void print_field(Microenvironment& M, const char* tag) {
  for (int n = 0; n < M.number_of_voxels(); ++n) {
    std::vector<double>& v = M.density_vector(n);
    for (size_t s = 0; s < v.size(); ++s) std::printf("%s %d %zu %.17g\n", tag, n, s, v[s]);
  }
}

static void print_gradients(Microenvironment& M, const char* tag, int stride) {
  for (int n = 0; n < M.number_of_voxels(); n += stride) {
    std::vector<gradient>& g = M.gradient_vector(n);
    for (size_t s = 0; s < g.size(); ++s)
      for (int c = 0; c < 3; ++c) std::printf("%s %d %zu %d %.17g\n", tag, n, s, c, g[s][c]);
  }
}

int main() {
  Microenvironment M;
  M.agent_container = new Agent_Container;  // the reference leaves it unset
  M.name = "api driver";
  M.set_density(0, "oxygen", "mmHg");
  M.add_density("glucose", "mM");
  M.resize_space_uniform(0.0, 200.0, 0.0, 160.0, 0.0, 120.0, 10.0);  // 20 x 16 x 12
  M.diffusion_coefficients[0] = 1.0e3;
  M.diffusion_coefficients[1] = 2.5e4;
  M.decay_rates[0] = 0.1;
  M.decay_rates[1] = 0.7;
  M.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
  for (int n = 0; n < M.number_of_voxels(); ++n) {
    const std::vector<double>& c = M.voxels(n).center;
    M.density_vector(n)[0] = 1.0 + std::sin(c[0] / 37.0) * std::cos(c[1] / 23.0);
    M.density_vector(n)[1] = 0.5 + c[2] / 240.0;
  }
  std::vector<double> dir_value(2);
  dir_value[0] = 3.0;
  dir_value[1] = 0.25;
  for (int j = 0; j < 16; j += 3) M.add_dirichlet_node(M.voxel_index(0, j, 5), dir_value);

  const double dt = 0.01;
  std::vector<Basic_Agent*> agents;
  for (int a = 0; a < 60; ++a) {
    Basic_Agent* p = create_basic_agent();
    p->register_microenvironment(&M);
    // several agents per voxel: the order of their updates matters
    p->assign_position(15.0 + 17.0 * (a % 9), 12.0 + 11.0 * (a % 7), 7.0 + 13.0 * (a % 5));
    p->volume = 1500.0 + 40.0 * a;
    p->secretion_rates->assign(2, 0.0);
    p->saturation_densities->assign(2, 1.0);
    p->uptake_rates->assign(2, 0.0);
    (*p->secretion_rates)[0] = 0.3 * (a % 4);
    (*p->uptake_rates)[1] = 0.05 * (a % 6);
    (*p->saturation_densities)[0] = 2.0;
    p->set_internal_uptake_constants(dt);
    agents.push_back(p);
  }
  for (int t = 0; t < 6; ++t) {
    M.simulate_cell_sources_and_sinks(dt);
    M.simulate_diffusion_decay(dt);
  }
  M.compute_all_gradient_vectors();
  print_gradients(M, "G", 1);
  print_field(M, "P");
  // the lazy path: after a reset, gradient_vector(n) computes voxel by voxel
  M.reset_all_gradient_vectors();
  M.density_vector(7)[0] += 0.5;  // a direct write between steps
  M.simulate_cell_sources_and_sinks(dt);
  M.simulate_diffusion_decay(dt);
  print_gradients(M, "L", 5);
  print_field(M, "Q");
  return 0;
}
