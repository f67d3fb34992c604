// Basic_Agent of the drop-in headers (BioFVM_basic_agent.cpp).  Compiled
// without FMA contraction: set_internal_uptake_constants reproduces the
// reference's constants bit for bit.
#include "BioFVM.h"

namespace BioFVM {

std::vector<Basic_Agent*> all_basic_agents(0);

namespace {
uint64_t g_epoch = 0;
}

uint64_t basic_agent_epoch(void) { return g_epoch; }
void touch_basic_agents(void) { ++g_epoch; }

Basic_Agent::Basic_Agent() {
  // BioFVM_basic_agent.cpp:37-56
  static int max_basic_agent_ID = 0;
  ID = max_basic_agent_ID++;
  index = -1;
  type = 0;
  volume = 2494.0;
  selected_microenvironment = 0;
  current_voxel_index = 0;
  position.assign(3, 0.0);
  velocity.assign(3, 0.0);
  previous_velocity.assign(3, 0.0);
  secretion_rates = new std::vector<double>(0);
  uptake_rates = new std::vector<double>(0);
  saturation_densities = new std::vector<double>(0);
  microenvironment = nullptr;
  if (get_default_microenvironment()) register_microenvironment(get_default_microenvironment());
}

Basic_Agent::~Basic_Agent() {
  delete secretion_rates;
  delete uptake_rates;
  delete saturation_densities;
}

void Basic_Agent::update_position(double) {}

void Basic_Agent::register_microenvironment(Microenvironment* M) {
  // BioFVM_basic_agent.cpp:150-161
  microenvironment = M;
  const size_t S = M->number_of_densities();
  secretion_rates->resize(S, 0.0);
  saturation_densities->resize(S, 0.0);
  uptake_rates->resize(S, 0.0);
  cell_source_sink_solver_temp1.resize(S, 0.0);
  cell_source_sink_solver_temp2.resize(S, 1.0);
  touch_basic_agents();
}

Microenvironment* Basic_Agent::get_microenvironment(void) { return microenvironment; }

bool Basic_Agent::assign_position(std::vector<double> p) {
  return assign_position(p[0], p[1], p[2]);
}

bool Basic_Agent::assign_position(double x, double y, double z) {
  // BioFVM_basic_agent.cpp:66-81: rejected outside the box, else the
  // nearest voxel is cached
  if (!microenvironment->mesh.is_position_valid(x, y, z)) return false;
  position[0] = x;
  position[1] = y;
  position[2] = z;
  current_voxel_index = microenvironment->nearest_voxel_index(position);
  touch_basic_agents();
  return true;
}

void Basic_Agent::set_internal_uptake_constants(double dt) {
  // BioFVM_basic_agent.cpp:122-147
  const double c = dt * volume / microenvironment->voxels(current_voxel_index).volume;
  const size_t S = secretion_rates->size();
  cell_source_sink_solver_temp1.assign(S, 0.0);
  cell_source_sink_solver_temp2.assign(S, 1.0);
  for (size_t s = 0; s < S; ++s) {
    double a = 0.0;
    a += (*secretion_rates)[s];
    a *= (*saturation_densities)[s];
    a *= c;
    cell_source_sink_solver_temp1[s] = a;
    double b = 1.0;
    b += c * (*secretion_rates)[s];
    b += c * (*uptake_rates)[s];
    cell_source_sink_solver_temp2[s] = b;
  }
  touch_basic_agents();
}

void Basic_Agent::simulate_secretion_and_uptake(Microenvironment* pS, double) {
  // BioFVM_basic_agent.cpp:234-235, on the host copy of this one voxel
  std::vector<double>& v = pS->density_vector(current_voxel_index);
  v += cell_source_sink_solver_temp1;
  v /= cell_source_sink_solver_temp2;
}

int Basic_Agent::nearest_voxel_index(void) { return current_voxel_index; }

std::vector<double>& Basic_Agent::nearest_density_vector(void) {
  return microenvironment->nearest_density_vector(current_voxel_index);
}

Basic_Agent* create_basic_agent(void) {
  // BioFVM_basic_agent.cpp:172-181
  Basic_Agent* p = new Basic_Agent;
  all_basic_agents.push_back(p);
  p->index = (int)all_basic_agents.size() - 1;
  touch_basic_agents();
  return p;
}

void delete_basic_agent(int index) {
  // BioFVM_basic_agent.cpp:183-204: the last agent moves into the hole
  delete all_basic_agents[index];
  all_basic_agents[index] = all_basic_agents.back();
  all_basic_agents[index]->index = index;
  all_basic_agents.pop_back();
  touch_basic_agents();
}

void delete_basic_agent(Basic_Agent* p) { delete_basic_agent(p->index); }

}  // namespace BioFVM
