// Basic_Agent with BioFVM's public API (BioFVM_basic_agent.h:40-95).  The
// secretion/uptake constants of set_internal_uptake_constants are computed on
// the host exactly as the reference does and sent to the device by the next
// simulate_cell_sources_and_sinks.
#ifndef __BioFVM_basic_agent_h__
#define __BioFVM_basic_agent_h__

#include <cstdint>
#include <string>
#include <vector>

#include "BioFVM_microenvironment.h"

namespace BioFVM {

class Basic_Agent {
 private:
  friend class Microenvironment;
  Microenvironment* microenvironment;
  int selected_microenvironment;
  std::vector<double> cell_source_sink_solver_temp1;
  std::vector<double> cell_source_sink_solver_temp2;

 protected:
  std::vector<double> previous_velocity;
  int current_voxel_index;

 public:
  std::vector<double>* secretion_rates;
  std::vector<double>* saturation_densities;
  std::vector<double>* uptake_rates;

  void set_internal_uptake_constants(double dt);

  void register_microenvironment(Microenvironment*);
  Microenvironment* get_microenvironment(void);

  int ID;
  int index;
  int type;
  double volume;

  bool assign_position(double x, double y, double z);
  bool assign_position(std::vector<double> new_position);

  std::vector<double> position;
  std::vector<double> velocity;
  void update_position(double dt);

  Basic_Agent();
  ~Basic_Agent();
  void simulate_secretion_and_uptake(Microenvironment* M, double dt);

  int nearest_voxel_index(void);
  std::vector<double>& nearest_density_vector(void);
};

extern std::vector<Basic_Agent*> all_basic_agents;

Basic_Agent* create_basic_agent(void);
void delete_basic_agent(int);
void delete_basic_agent(Basic_Agent*);

// Incremented whenever an agent's voxel or secretion/uptake constants change
// or agents are created / deleted; the device copy is refreshed when it moves.
uint64_t basic_agent_epoch(void);
void touch_basic_agents(void);

}  // namespace BioFVM

#endif
