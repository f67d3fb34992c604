// The reference's Agent_Container is a set of empty stubs
// (BioFVM_agent_container.cpp:37-47); kept so that driver code that names it
// compiles.
#ifndef __BioFVM_agent_container_h__
#define __BioFVM_agent_container_h__

#include <vector>

namespace BioFVM {
class Basic_Agent;
class Agent_Container {
 public:
  std::vector<std::vector<Basic_Agent*> > agent_grid;
  Agent_Container() {}
  void register_agent(Basic_Agent*) {}
  void initialize(int) {}
  void remove_agent(Basic_Agent*) {}
};
}  // namespace BioFVM

#endif
