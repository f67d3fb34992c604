// MATLAB Level-4 matrix files with BioFVM's names (BioFVM_matlab.h): the
// reference's only output format.  Real, full, double matrices only.
#ifndef __BioFVM_matlab_h__
#define __BioFVM_matlab_h__

#include <cstdio>
#include <string>
#include <vector>

namespace BioFVM {
struct named_vector_data {
  std::vector<std::string> names;
  std::vector<std::vector<double> > data;
};
std::vector<std::vector<double> > read_matlab(std::string filename);
bool write_matlab(std::vector<std::vector<double> >& input, std::string filename);
FILE* write_matlab_header(int rows, int cols, std::string filename, std::string variable_name);
FILE* read_matlab_header(int* rows, int* cols, std::string filename);
}  // namespace BioFVM

#endif
