// Solver entry points with BioFVM's names (BioFVM_solvers.h).  The LOD_3D
// solver runs on the GPU (libbfvm.so); it is also what
// Microenvironment::diffusion_decay_solver points to by default.
#ifndef __BioFVM_solvers_h__
#define __BioFVM_solvers_h__

#include "BioFVM_microenvironment.h"

namespace BioFVM {
void diffusion_decay_solver__constant_coefficients_LOD_3D(Microenvironment& M, double dt);
void diffusion_decay_solver__constant_coefficients_LOD_2D(Microenvironment& M, double dt);
void diffusion_decay_explicit_uniform_rates(Microenvironment& M, double dt);
void diffusion_decay_solver__constant_coefficients_explicit(Microenvironment& M, double dt);
void diffusion_decay_solver__constant_coefficients_explicit_uniform_mesh(Microenvironment& M,
                                                                          double dt);
}  // namespace BioFVM

#endif
