// Host-side Cartesian mesh with BioFVM's names (BioFVM_mesh.h:49-188):
// voxel centres, volumes, indices and nearest-voxel lookup by the reference's
// formulas, and each voxel's list of face-connected neighbours.  Only the
// Cartesian mesh of the transport path is provided; voxel faces (unused by
// the LOD solver) are not built.
#ifndef __BioFVM_mesh_h__
#define __BioFVM_mesh_h__

#include <iostream>
#include <string>
#include <vector>

namespace BioFVM {

class Voxel {
 public:
  Voxel();
  int mesh_index;
  double volume;
  std::vector<double> center;
  bool is_Dirichlet;
};

std::ostream& operator<<(std::ostream& os, const Voxel& v);

class General_Mesh {
 public:
  General_Mesh();
  std::vector<double> bounding_box;  // [xmin ymin zmin xmax ymax zmax]
  std::vector<Voxel> voxels;
  // per voxel its face neighbours, in the order the reference connects them
  // (BioFVM_mesh.cpp:873-915): x-1, x+1, y-1, y+1, z-1, z+1 where present
  std::vector<std::vector<int> > connected_voxel_indices;
  bool is_position_valid(double x, double y, double z);
  // adds j to voxel i's list and i to voxel j's (BioFVM_mesh.cpp:260-268)
  void connect_voxels_indices_only(int i, int j, double SA);
  bool Cartesian_mesh;
  bool uniform_mesh;
  bool regular_mesh;
  bool use_voxel_faces;
  std::string units;
  void display_information(std::ostream& os);
  // [4][voxels] MATLAB matrix "mesh": centre x, y, z and volume per voxel
  // (BioFVM_mesh.cpp:350-367)
  void write_to_matlab(std::string filename);
};

class Cartesian_Mesh : public General_Mesh {
 public:
  std::vector<double> x_coordinates;
  std::vector<double> y_coordinates;
  std::vector<double> z_coordinates;
  int voxel_index(int i, int j, int k);
  std::vector<int> cartesian_indices(int n);
  double dx, dy, dz;
  double dV, dS;
  double dS_xy, dS_yz, dS_xz;

  Cartesian_Mesh();
  Cartesian_Mesh(int xnodes, int ynodes, int znodes);
  void resize(int x_nodes, int y_nodes, int z_nodes);
  void resize(double x_start, double x_end, double y_start, double y_end, double z_start,
              double z_end, int x_nodes, int y_nodes, int z_nodes);
  void resize(double x_start, double x_end, double y_start, double y_end, double z_start,
              double z_end, double dx, double dy, double dz);
  void resize_uniform(double x_start, double x_end, double y_start, double y_end,
                      double z_start, double z_end, double dx);
  int nearest_voxel_index(std::vector<double>& position);
  std::vector<int> nearest_cartesian_indices(std::vector<double>& position);
  Voxel& nearest_voxel(std::vector<double>& position);
  void display_information(std::ostream& os);

 private:
  void build_voxels();
};

}  // namespace BioFVM

#endif
