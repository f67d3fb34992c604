// A driver of the MultiCellDS save/load API for the drop-in test: built once
// against the reference sources and once against biofvm_b200's headers.  It
// saves a small microenvironment (data as MATLAB files or inline XML, mesh as
// coordinates or voxel lists), saves again after a change (the second save
// updates the time and the data of the document already built), and reads a
// saved file back into a new microenvironment, printing what it reads.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "BioFVM.h"
#include "BioFVM_MultiCellDS.h"

using namespace BioFVM;

static void print_env(Microenvironment& M, const char* tag) {
  std::printf("%s name %s units %s\n", tag, M.name.c_str(), M.mesh.units.c_str());
  std::printf("%s shape %zu %zu %zu voxels %d\n", tag, M.mesh.x_coordinates.size(),
              M.mesh.y_coordinates.size(), M.mesh.z_coordinates.size(), M.number_of_voxels());
  for (int s = 0; s < M.number_of_densities(); ++s)
    std::printf("%s density %d %s %s %.17g %.17g\n", tag, s, M.density_names[s].c_str(),
                M.density_units[s].c_str(), M.diffusion_coefficients[s], M.decay_rates[s]);
  for (int n = 0; n < M.number_of_voxels(); ++n) {
    std::vector<double>& v = M.density_vector(n);
    for (size_t s = 0; s < v.size(); ++s) std::printf("%s p %d %zu %.17g\n", tag, n, s, v[s]);
  }
}

int main(int argc, char** argv) {
  const bool data_matlab = argc > 1 && std::strcmp(argv[1], "1") == 0;
  const bool mesh_matlab = argc > 2 && std::strcmp(argv[2], "1") == 0;
  Microenvironment M;
  M.name = "mcds test";
  M.set_density(0, "oxygen", "mmHg");
  M.add_density("glucose", "mM");
  M.spatial_units = "microns";
  M.mesh.units = "microns";
  M.resize_space_uniform(0.0, 60.0, 0.0, 40.0, 0.0, 30.0, 10.0);  // 6 x 4 x 3
  M.diffusion_coefficients[0] = 1.0e5;
  M.diffusion_coefficients[1] = 1234.5;
  M.decay_rates[0] = 0.1;
  M.decay_rates[1] = 0.015625;
  for (int n = 0; n < M.number_of_voxels(); ++n) {
    M.density_vector(n)[0] = 0.5 + 0.25 * n;
    M.density_vector(n)[1] = 38.0 - 0.125 * n;
  }
  default_metadata.user = "driver";
  default_metadata.current_time = 1.5;
  default_metadata.current_runtime = 0.25;
  set_save_biovm_data_as_matlab(data_matlab);
  set_save_biovm_mesh_as_matlab(mesh_matlab);
  save_microenvironment_to_MultiCellDS_xml_pugi("first", M);
  M.density_vector(0)[0] = 7.0;
  default_metadata.current_time = 2.5;
  save_microenvironment_to_MultiCellDS_xml_pugi("second", M);

  Microenvironment R;
  read_microenvironment_from_MultiCellDS_xml(R, "first.xml");
  print_env(R, "R");
  return 0;
}
