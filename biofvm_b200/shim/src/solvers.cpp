// Solver entry points of the drop-in headers (BioFVM_solvers.cpp).
#include "BioFVM.h"
#include "bfvm.h"

namespace BioFVM {

void diffusion_decay_solver__constant_coefficients_LOD_3D(Microenvironment& M, double dt) {
  // BioFVM_solvers.cpp:77-276 on the GPU; the reference prints this banner
  // on its first call (:89-90)
  static bool announced = false;
  if (!announced) {
    std::cout << std::endl
              << "Using method diffusion_decay_solver__constant_coefficients_LOD_3D "
                 "(implicit 3-D LOD with Thomas Algorithm) ... "
              << std::endl
              << std::endl;
    announced = true;
  }
  M.prepare_step(false, false, nullptr);
  const int rc = bfvm_simulate_diffusion_decay(M.solver_, dt);
  if (rc == BFVM_ERR_MESH) {  // :79-83
    std::cout << "Error: This algorithm is written for uniform Cartesian meshes. Try: other "
                 "solvers!"
              << std::endl
              << std::endl;
    return;
  }
  if (rc != BFVM_OK) throw std::runtime_error(std::string("LOD_3D: ") + bfvm_last_error());
  M.host_valid_.store(false);
}

void diffusion_decay_solver__constant_coefficients_LOD_2D(Microenvironment& M, double dt) {
  static bool announced = false;
  if (!announced) {
    std::cout << std::endl
              << "Using method diffusion_decay_solver__constant_coefficients_LOD_2D "
                 "(implicit 2-D LOD with Thomas Algorithm) ... "
              << std::endl
              << std::endl;
    announced = true;
  }
  M.prepare_step(false, false, nullptr);
  const int rc = bfvm_simulate_diffusion_decay_2d(M.solver_, dt);
  if (rc == BFVM_ERR_MESH) {
    std::cout << "Error: This algorithm is written for uniform Cartesian meshes. Try: "
                 "something else."
              << std::endl
              << std::endl;
    return;
  }
  if (rc != BFVM_OK) throw std::runtime_error(std::string("LOD_2D: ") + bfvm_last_error());
  M.host_valid_.store(false);
}

// The reference's explicit solvers (BioFVM_solvers.cpp:38-74) only announce
// themselves and return; kept with the same behaviour.
void diffusion_decay_solver__constant_coefficients_explicit(Microenvironment& M, double) {
  static bool done = false;
  if (!done) {
    std::cout << std::endl
              << "Using solver: diffusion_decay_solver__constant_coefficients_explicit"
              << std::endl
              << "     (constant diffusion coefficient with explicit stepping, implicit "
                 "decay) ... "
              << std::endl
              << std::endl;
    if (M.mesh.uniform_mesh)
      std::cout << "Uniform mesh detected! Consider switching to a more efficient method, such "
                   "as "
                << std::endl
                << "     diffusion_decay_solver__constant_coefficients_explicit_uniform_mesh"
                << std::endl
                << std::endl;
    done = true;
  }
}

void diffusion_decay_solver__constant_coefficients_explicit_uniform_mesh(Microenvironment& M,
                                                                          double) {
  static bool done = false;
  if (!done) {
    std::cout << std::endl
              << "Using solver: "
                 "diffusion_decay_solver__constant_coefficients_explicit_uniform_mesh"
              << std::endl
              << "     (constant diffusion coefficient with explicit stepping, implicit "
                 "decay, uniform mesh) ... "
              << std::endl
              << std::endl;
    if (!M.mesh.uniform_mesh)
      std::cout << "Error. This code is only supported for uniform meshes." << std::endl;
    done = true;
  }
}

// The reference's explicit uniform-rate solver (BioFVM_solvers.cpp:429-497)
// is not part of the transport path built here.
void diffusion_decay_explicit_uniform_rates(Microenvironment&, double) {
  std::cout << "diffusion_decay_explicit_uniform_rates is not available in this build; use "
               "diffusion_decay_solver__constant_coefficients_LOD_3D"
            << std::endl;
}

}  // namespace BioFVM
