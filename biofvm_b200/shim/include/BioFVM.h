// Drop-in replacement of BioFVM's umbrella header for the B200 transport
// path: same header names, namespace and public API as BioFVM 1.0.4
// (BioFVM.h), implemented over the C ABI of libbfvm.so (include/bfvm.h).
#ifndef __BioFVM_h__
#define __BioFVM_h__

#include <fstream>
#include <iostream>
#include <string>

namespace BioFVM {
extern std::string BioFVM_Version;
extern std::string BioFVM_URL;
}  // namespace BioFVM

#include "BioFVM_utilities.h"
#include "BioFVM_vector.h"
#include "BioFVM_mesh.h"
#include "BioFVM_microenvironment.h"
#include "BioFVM_solvers.h"
#include "BioFVM_basic_agent.h"
#include "BioFVM_matlab.h"

#endif
