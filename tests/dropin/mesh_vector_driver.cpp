// Host-side parts of the BioFVM API for the drop-in test, built once against
// the reference sources and once against biofvm_b200's headers: the mesh's
// voxel connectivity lists and the CSV helpers of BioFVM_vector.h.  Prints
// every value, one per line, for the test to compare.  Built against the
// drop-in headers (DROPIN_SHIM) it also prints the fused elementwise helpers
// that the reference declares but does not define.
#include <cstdio>
#include <vector>

#include "BioFVM.h"

using namespace BioFVM;

static void print_connectivity(Cartesian_Mesh& m, const char* tag) {
  std::printf("%s size %zu\n", tag, m.connected_voxel_indices.size());
  for (size_t n = 0; n < m.connected_voxel_indices.size(); ++n) {
    std::printf("%s %zu:", tag, n);
    for (int v : m.connected_voxel_indices[n]) std::printf(" %d", v);
    std::printf("\n");
  }
}

int main() {
  Cartesian_Mesh a;
  print_connectivity(a, "C0");  // the default one-voxel mesh
  a.resize(0.0, 70.0, 0.0, 50.0, 0.0, 40.0, 10.0, 10.0, 10.0);  // 7 x 5 x 4
  print_connectivity(a, "C1");
  Cartesian_Mesh b;
  b.resize(0.0, 30.0, 0.0, 10.0, 0.0, 20.0, 3, 1, 2);  // a one-node axis
  print_connectivity(b, "C2");

  std::vector<double> v = {1.0, -2.5e-7, 3.14159265358979, 6.02e23, -0.0, 1e-300};
  char* s1 = vector_to_csv(v);
  std::printf("S1 %s\n", s1);
  delete[] s1;
  char* s2 = nullptr;
  vector_to_csv_safe(v, s2);
  vector_to_csv_safe(v, s2);  // replaces its own buffer
  std::printf("S2 %s\n", s2);
  delete[] s2;
  char* s3 = new char[16 * v.size() + 1];
  vector_to_csv(v, s3);
  std::printf("S3 %s\n", s3);
  std::vector<double> back;
  csv_to_vector(s3, back);
  for (double x : back) std::printf("B %.17g\n", x);
  delete[] s3;

#ifdef DROPIN_SHIM
  std::vector<double> y = {1.0, 2.0, 3.0}, a1 = {0.5, -1.0, 2.0}, a2 = {3.0, 0.25, -0.5},
                      x1 = {4.0, 5.0, -6.0}, x2 = {-1.0, 2.0, 0.125}, d = {2.0, 4.0, -8.0};
  std::vector<double> t = y;
  axpy_div(&t, a1, x1, d);
  for (double q : t) std::printf("V axpy_div %.17g\n", q);
  t = y;
  double_axpy(&t, a1, a2, x1, x2);
  for (double q : t) std::printf("V double_axpy2 %.17g\n", q);
  t = y;
  double_axpy(&t, a1, x1, x2);
  for (double q : t) std::printf("V double_axpy1 %.17g\n", q);
  t = y;
  double_axpy_div(&t, a1, x1, x2, d);
  for (double q : t) std::printf("V double_axpy_div1 %.17g\n", q);
  t = y;
  double_axpy_div(&t, a1, a2, x1, x2, d);
  for (double q : t) std::printf("V double_axpy_div2 %.17g\n", q);
#endif
  return 0;
}
