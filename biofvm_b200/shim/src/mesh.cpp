// Cartesian mesh geometry of the drop-in headers: node counts, centres,
// volumes and nearest-voxel lookup by the formulas of BioFVM_mesh.cpp
// (:663-948), computed without FMA contraction so that agents land in the
// reference's voxels.
#include <cmath>

#include "BioFVM_mesh.h"
#include "BioFVM_matlab.h"

namespace BioFVM {

Voxel::Voxel() : mesh_index(0), volume(10.0 * 10.0 * 10.0), center(3, 0.0), is_Dirichlet(false) {}

std::ostream& operator<<(std::ostream& os, const Voxel& v) {
  os << "I am voxel #" << v.mesh_index << " centered at " << v.center[0] << " " << v.center[1]
     << " " << v.center[2] << " with volume " << v.volume;
  return os;
}

General_Mesh::General_Mesh()
    : bounding_box{-0.5, -0.5, -0.5, 0.5, 0.5, 0.5},
      voxels(1),
      connected_voxel_indices(1),
      Cartesian_mesh(false),
      uniform_mesh(false),
      regular_mesh(false),
      use_voxel_faces(false),
      units("none") {}

void General_Mesh::connect_voxels_indices_only(int i, int j, double) {
  connected_voxel_indices[i].push_back(j);
  connected_voxel_indices[j].push_back(i);
}

bool General_Mesh::is_position_valid(double x, double y, double z) {
  // BioFVM_mesh.cpp:208-217
  return !(x < bounding_box[0] || x > bounding_box[3] || y < bounding_box[1] ||
           y > bounding_box[4] || z < bounding_box[2] || z > bounding_box[5]);
}

void General_Mesh::write_to_matlab(std::string filename) {
  FILE* fp = write_matlab_header(4, (int)voxels.size(), filename, "mesh");
  if (!fp) return;
  for (const Voxel& v : voxels) {
    const double col[4] = {v.center[0], v.center[1], v.center[2], v.volume};
    std::fwrite(col, sizeof(double), 4, fp);
  }
  std::fclose(fp);
}

void General_Mesh::display_information(std::ostream& os) {
  os << "Mesh information: " << std::endl
     << "   voxels: " << voxels.size() << std::endl
     << "   bounding box: [" << bounding_box[0] << "," << bounding_box[3] << "] x ["
     << bounding_box[1] << "," << bounding_box[4] << "] x [" << bounding_box[2] << ","
     << bounding_box[5] << "] " << units << std::endl;
}

Cartesian_Mesh::Cartesian_Mesh() {
  Cartesian_mesh = true;
  resize(1, 1, 1);
}

Cartesian_Mesh::Cartesian_Mesh(int xnodes, int ynodes, int znodes) {
  Cartesian_mesh = true;
  resize(xnodes, ynodes, znodes);
}

int Cartesian_Mesh::voxel_index(int i, int j, int k) {
  return (k * (int)y_coordinates.size() + j) * (int)x_coordinates.size() + i;
}

std::vector<int> Cartesian_Mesh::cartesian_indices(int n) {
  const int nx = (int)x_coordinates.size(), ny = (int)y_coordinates.size();
  std::vector<int> out(3);
  out[2] = n / (nx * ny);
  out[1] = (n - out[2] * nx * ny) / nx;
  out[0] = n - nx * (out[1] + ny * out[2]);
  return out;
}

void Cartesian_Mesh::build_voxels() {
  dV = dx * dy * dz;
  dS = dx * dy;
  dS_xy = dx * dy;
  dS_yz = dy * dz;
  dS_xz = dx * dz;
  const size_t nx = x_coordinates.size(), ny = y_coordinates.size(), nz = z_coordinates.size();
  Voxel tpl;
  tpl.volume = dV;
  voxels.assign(nx * ny * nz, tpl);
  size_t n = 0;
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i, ++n) {
        Voxel& v = voxels[n];
        v.center[0] = x_coordinates[i];
        v.center[1] = y_coordinates[j];
        v.center[2] = z_coordinates[k];
        v.mesh_index = (int)n;
        v.volume = dV;
      }
  // the reference connects all x pairs, then all y pairs, then all z pairs,
  // each pair (lower, upper) once, so every voxel's list reads x-1, x+1,
  // y-1, y+1, z-1, z+1 (those that exist)
  connected_voxel_indices.assign(nx * ny * nz, std::vector<int>());
  const int jx = 1, jy = (int)nx, jz = (int)(nx * ny);
  n = 0;
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i, ++n) {
        std::vector<int>& c = connected_voxel_indices[n];
        const int v = (int)n;
        c.reserve(6);
        if (i > 0) c.push_back(v - jx);
        if (i + 1 < nx) c.push_back(v + jx);
        if (j > 0) c.push_back(v - jy);
        if (j + 1 < ny) c.push_back(v + jy);
        if (k > 0) c.push_back(v - jz);
        if (k + 1 < nz) c.push_back(v + jz);
      }
}

void Cartesian_Mesh::resize(double x0, double x1, double y0, double y1, double z0, double z1,
                            int nx, int ny, int nz) {
  // BioFVM_mesh.cpp:663-704: spacing from the node counts; a single node has
  // spacing 1
  dx = (x1 - x0) / (double)nx;
  if (nx < 2) dx = 1;
  dy = (y1 - y0) / (double)ny;
  if (ny < 2) dy = 1;
  dz = (z1 - z0) / (double)nz;
  if (nz < 2) dz = 1;
  const double tol = 1e-16;
  uniform_mesh = true;
  regular_mesh = true;
  if (std::fabs(dx - dy) > tol && nx > 1 && ny > 1) uniform_mesh = false;
  if (std::fabs(dy - dz) > tol && ny > 1 && nz > 1) uniform_mesh = false;
  if (std::fabs(dx - dz) > tol && nx > 1 && nz > 1) uniform_mesh = false;
  x_coordinates.assign(nx, 0.0);
  y_coordinates.assign(ny, 0.0);
  z_coordinates.assign(nz, 0.0);
  for (int i = 0; i < nx; ++i) x_coordinates[i] = x0 + (i + 0.5) * dx;
  for (int i = 0; i < ny; ++i) y_coordinates[i] = y0 + (i + 0.5) * dy;
  for (int i = 0; i < nz; ++i) z_coordinates[i] = z0 + (i + 0.5) * dz;
  bounding_box = {x0, y0, z0, x1, y1, z1};
  build_voxels();
}

void Cartesian_Mesh::resize(double x0, double x1, double y0, double y1, double z0, double z1,
                            double dx_new, double dy_new, double dz_new) {
  // BioFVM_mesh.cpp:796-836: node counts ceil(1e-16 + L/d)
  dx = dx_new;
  dy = dy_new;
  dz = dz_new;
  const double eps = 1e-16;
  const int nx = (int)std::ceil(eps + (x1 - x0) / dx);
  const int ny = (int)std::ceil(eps + (y1 - y0) / dy);
  const int nz = (int)std::ceil(eps + (z1 - z0) / dz);
  const double tol = 1e-16;
  uniform_mesh = !(std::fabs(dx - dy) > tol || std::fabs(dy - dz) > tol ||
                   std::fabs(dx - dz) > tol);
  regular_mesh = true;
  x_coordinates.assign(nx, 0.0);
  y_coordinates.assign(ny, 0.0);
  z_coordinates.assign(nz, 0.0);
  for (int i = 0; i < nx; ++i) x_coordinates[i] = x0 + (i + 0.5) * dx;
  for (int i = 0; i < ny; ++i) y_coordinates[i] = y0 + (i + 0.5) * dy;
  for (int i = 0; i < nz; ++i) z_coordinates[i] = z0 + (i + 0.5) * dz;
  bounding_box = {x0, y0, z0, x1, y1, z1};
  build_voxels();
}

void Cartesian_Mesh::resize(int nx, int ny, int nz) {
  // BioFVM_mesh.cpp:924-925: unit spacing centred on the integer nodes
  resize(0 - .5, nx - 1 + .5, 0 - .5, ny - 1 + .5, 0 - .5, nz - 1 + .5, nx, ny, nz);
}

void Cartesian_Mesh::resize_uniform(double x0, double x1, double y0, double y1, double z0,
                                    double z1, double d) {
  resize(x0, x1, y0, y1, z0, z1, d, d, d);
}

std::vector<int> Cartesian_Mesh::nearest_cartesian_indices(std::vector<double>& position) {
  // BioFVM_mesh.cpp:930-947: floor((x - min)/d), clamped to the mesh
  const int nx = (int)x_coordinates.size(), ny = (int)y_coordinates.size(),
            nz = (int)z_coordinates.size();
  std::vector<int> out(3);
  out[0] = (int)std::floor((position[0] - bounding_box[0]) / dx);
  out[1] = (int)std::floor((position[1] - bounding_box[1]) / dy);
  out[2] = (int)std::floor((position[2] - bounding_box[2]) / dz);
  const int lim[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    if (out[a] >= lim[a]) out[a] = lim[a] - 1;
    if (out[a] < 0) out[a] = 0;
  }
  return out;
}

int Cartesian_Mesh::nearest_voxel_index(std::vector<double>& position) {
  const std::vector<int> c = nearest_cartesian_indices(position);
  return voxel_index(c[0], c[1], c[2]);
}

Voxel& Cartesian_Mesh::nearest_voxel(std::vector<double>& position) {
  return voxels[nearest_voxel_index(position)];
}

void Cartesian_Mesh::display_information(std::ostream& os) {
  os << std::endl
     << "Mesh information: " << std::endl
     << "type: uniform Cartesian" << std::endl
     << "Domain: [" << bounding_box[0] << "," << bounding_box[3] << "] " << units << " x ["
     << bounding_box[1] << "," << bounding_box[4] << "] " << units << " x [" << bounding_box[2]
     << "," << bounding_box[5] << "] " << units << std::endl
     << "   resolution: dx = " << dx << " " << units << std::endl
     << "   voxels: " << voxels.size() << std::endl
     << "   voxel faces: 0" << std::endl
     << "   volume: "
     << (bounding_box[3] - bounding_box[0]) * (bounding_box[4] - bounding_box[1]) *
            (bounding_box[5] - bounding_box[2])
     << " cubic " << units << std::endl;
}

}  // namespace BioFVM
