// MultiCellDS snapshots with BioFVM's names (BioFVM_MultiCellDS.h:30-88):
// save a Microenvironment to a MultiCellDS XML file (densities inline or in
// a MATLAB file, mesh as coordinates plus a voxel list inline or in a MATLAB
// file) and read one back.  The document is written and parsed by this
// library's own small XML code: the reference's pugixml DOM types
// (pugi::xml_document, the DOM overload of the reader, biofvm_doc) are not
// offered.
#ifndef __BioFVM_MultiCellDS_h__
#define __BioFVM_MultiCellDS_h__

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace BioFVM {
extern std::string MultiCellDS_version_string;
extern std::string MultiCellDS_experimental_snapshot_type_string;
extern int MultiCellDS_experimental_snapshot_code;

extern std::string MultiCellDS_simulation_snapshot_type_string;
extern int MultiCellDS_simulation_snapshot_code;

extern std::string MultiCellDS_digital_cell_line_type_string;
extern int MultiCellDS_digital_cell_line_code;

extern std::string MultiCellDS_generic_type_string;
extern int MultiCellDS_generic_code;

class Microenvironment;

class MultiCellDS_Metadata {
 public:
  std::string MultiCellDS_type;

  std::string user;
  std::string program;
  std::string program_version;

  std::vector<double> bounding_box;
  std::string spatial_units;
  std::string time_units;
  std::string runtime_time_units;
  double current_time;
  double current_runtime;

  MultiCellDS_Metadata();
  // declared by the reference without a definition; kept for source
  // compatibility (a call does not link, as with the reference)
  void add_to_open_MultiCellDS_xml(std::ostream& os, std::string base_tabbing);
};

extern MultiCellDS_Metadata default_metadata;

void read_microenvironment_from_MultiCellDS_xml(Microenvironment& M_destination,
                                                std::string filename);

void set_save_biovm_mesh_as_matlab(bool newvalue);
void set_save_biovm_data_as_matlab(bool newvalue);

void save_microenvironment_to_MultiCellDS_xml_pugi(std::string filename_base, Microenvironment& M);
}  // namespace BioFVM

#endif
