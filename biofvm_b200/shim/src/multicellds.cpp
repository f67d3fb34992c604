// MultiCellDS save/load of the drop-in headers (BioFVM_MultiCellDS.cpp).
//
// The document is held as a small tree of elements and written in the
// layout the reference's XML library produces by default (XML declaration,
// one element per line, tab indentation, text-only elements on one line), so
// that files written here and by the reference are the same text.  The
// reader is a small XML parser sufficient for these documents (elements,
// attributes, text, comments, the five predefined entities).
#include "BioFVM_MultiCellDS.h"

#include <cctype>
#include <cstdarg>
#include <fstream>
#include <sstream>

#include "BioFVM_matlab.h"
#include "BioFVM_microenvironment.h"
#include "BioFVM_vector.h"

namespace BioFVM {

std::string MultiCellDS_version_string = "0.3.0 beta";
std::string MultiCellDS_experimental_snapshot_type_string = "snapshot/experimental";
int MultiCellDS_experimental_snapshot_code = 3;
std::string MultiCellDS_simulation_snapshot_type_string = "snapshot/simulation";
int MultiCellDS_simulation_snapshot_code = 2;
std::string MultiCellDS_digital_cell_line_type_string = "digital_cell_line";
int MultiCellDS_digital_cell_line_code = 1;
std::string MultiCellDS_generic_type_string = "generic";
int MultiCellDS_generic_code = 0;

MultiCellDS_Metadata::MultiCellDS_Metadata()
    : MultiCellDS_type(MultiCellDS_generic_type_string),
      user("Unspecified"),
      program("BioFVM"),
      program_version("1.0.4"),
      bounding_box(6, 0.0),
      spatial_units("microns"),
      time_units("min"),
      runtime_time_units("seconds"),
      current_time(0.0),
      current_runtime(0.0) {}

MultiCellDS_Metadata default_metadata;

namespace {

// defaults of the reference (BioFVM_MultiCellDS.cpp:50-51)
bool save_mesh_as_matlab = false;
bool save_density_data_as_matlab = true;

struct XNode {
  std::string name;
  std::vector<std::pair<std::string, std::string> > attrs;
  std::string text;  // a text-only element
  std::vector<XNode> kids;

  XNode& add(const std::string& n) {
    kids.push_back(XNode());
    kids.back().name = n;
    return kids.back();
  }
  XNode& attr(const std::string& k, const std::string& v) {
    attrs.emplace_back(k, v);
    return *this;
  }
  XNode* child(const std::string& n) {
    for (auto& k : kids)
      if (k.name == n) return &k;
    return nullptr;
  }
  const char* value(const std::string& k) const {
    for (auto& a : attrs)
      if (a.first == k) return a.second.c_str();
    return "";
  }
  bool has(const std::string& k) const {
    for (auto& a : attrs)
      if (a.first == k) return true;
    return false;
  }
  void set(const std::string& k, const std::string& v) {
    for (auto& a : attrs)
      if (a.first == k) {
        a.second = v;
        return;
      }
    attrs.emplace_back(k, v);
  }
};

// The document of the last save: later saves update its time and data only,
// as the reference does with its global document (:401-470).
XNode g_doc;
bool g_doc_built = false;

std::string fmt(const char* f, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, f);
  std::vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}

std::string escape(const std::string& s, bool attribute) {
  std::string o;
  for (char c : s) {
    switch (c) {
      case '&': o += "&amp;"; break;
      case '<': o += "&lt;"; break;
      case '>': o += "&gt;"; break;
      case '"':
        if (attribute)
          o += "&quot;";
        else
          o += c;
        break;
      default: o += c;
    }
  }
  return o;
}

void write_node(std::ostream& os, const XNode& n, int depth) {
  const std::string tabs(depth, '\t');
  os << tabs << '<' << n.name;
  for (auto& a : n.attrs) os << ' ' << a.first << "=\"" << escape(a.second, true) << '"';
  if (n.kids.empty()) {
    if (n.text.empty())
      os << " />\n";
    else
      os << '>' << escape(n.text, false) << "</" << n.name << ">\n";
    return;
  }
  os << ">\n";
  for (auto& k : n.kids) write_node(os, k, depth + 1);
  os << tabs << "</" << n.name << ">\n";
}

std::string csv_of(const std::vector<double>& v, const char* f) {
  std::string s;
  for (size_t i = 0; i < v.size(); ++i) {
    if (i) s += ',';
    s += fmt(f, v[i]);
  }
  return s;
}

std::string bool_text(bool b) { return b ? "true" : "false"; }

// ---- the reader -------------------------------------------------------

struct Parser {
  const std::string& s;
  size_t i = 0;
  explicit Parser(const std::string& str) : s(str) {}

  static std::string decode(const std::string& t) {
    std::string o;
    for (size_t k = 0; k < t.size(); ++k) {
      if (t[k] != '&') {
        o += t[k];
        continue;
      }
      const size_t e = t.find(';', k);
      const std::string ent = t.substr(k + 1, e == std::string::npos ? 0 : e - k - 1);
      if (ent == "amp") o += '&';
      else if (ent == "lt") o += '<';
      else if (ent == "gt") o += '>';
      else if (ent == "quot") o += '"';
      else if (ent == "apos") o += '\'';
      else {
        o += '&';
        continue;
      }
      k = e;
    }
    return o;
  }
  void skip_misc() {
    for (;;) {
      while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
      if (s.compare(i, 4, "<!--") == 0) {
        const size_t e = s.find("-->", i);
        i = (e == std::string::npos) ? s.size() : e + 3;
      } else if (s.compare(i, 2, "<?") == 0) {
        const size_t e = s.find("?>", i);
        i = (e == std::string::npos) ? s.size() : e + 2;
      } else {
        return;
      }
    }
  }
  bool element(XNode& n) {
    skip_misc();
    if (i >= s.size() || s[i] != '<') return false;
    ++i;
    size_t b = i;
    while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/') ++i;
    n.name = s.substr(b, i - b);
    for (;;) {
      while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
      if (i >= s.size()) return false;
      if (s[i] == '/') {  // self-closing
        i = s.find('>', i) + 1;
        return true;
      }
      if (s[i] == '>') {
        ++i;
        break;
      }
      b = i;
      while (i < s.size() && s[i] != '=' && !std::isspace((unsigned char)s[i])) ++i;
      const std::string key = s.substr(b, i - b);
      i = s.find_first_of("\"'", i);
      if (i == std::string::npos) return false;
      const char q = s[i++];
      b = i;
      i = s.find(q, i);
      if (i == std::string::npos) return false;
      n.attrs.emplace_back(key, decode(s.substr(b, i - b)));
      ++i;
    }
    // content: text and child elements until the closing tag
    std::string text;
    for (;;) {
      if (i >= s.size()) return false;
      if (s.compare(i, 2, "</") == 0) {
        i = s.find('>', i) + 1;
        break;
      }
      if (s.compare(i, 4, "<!--") == 0) {
        const size_t e = s.find("-->", i);
        i = (e == std::string::npos) ? s.size() : e + 3;
        continue;
      }
      if (s[i] == '<') {
        n.kids.push_back(XNode());
        if (!element(n.kids.back())) return false;
        continue;
      }
      const size_t e = s.find('<', i);
      text += s.substr(i, (e == std::string::npos ? s.size() : e) - i);
      i = (e == std::string::npos) ? s.size() : e;
    }
    if (n.kids.empty()) n.text = decode(text);
    return true;
  }
};

// pugixml's as_bool: true when the value starts with 1, t, T, y or Y
bool as_bool(const char* v) {
  return v && (v[0] == '1' || v[0] == 't' || v[0] == 'T' || v[0] == 'y' || v[0] == 'Y');
}

void build_document(const std::string& filename_base, Microenvironment& M) {
  XNode root;
  root.name = "MultiCellDS";
  root.attr("version", MultiCellDS_version_string);
  root.attr("type", MultiCellDS_simulation_snapshot_type_string);
  XNode& md = root.add("metadata");
  md.add("user").text = default_metadata.user;
  {
    XNode& p = md.add("program");
    p.attr("version", default_metadata.program_version);
    p.text = default_metadata.program;
  }
  {
    XNode& bb = md.add("bounding_box");
    bb.attr("type", "axis-aligned").attr("units", default_metadata.spatial_units);
    const std::vector<double>& b = default_metadata.bounding_box;
    bb.text = fmt("[%f %f %f %f %f %f]", b[0], b[1], b[2], b[3], b[4], b[5]);
  }
  {
    XNode& t = md.add("current_time");
    t.attr("units", default_metadata.time_units);
    t.text = fmt("%f", default_metadata.current_time);
  }
  {
    XNode& t = md.add("current_runtime");
    t.attr("units", default_metadata.runtime_time_units);
    t.text = fmt("%f", default_metadata.current_runtime);
  }
  XNode& scale = root.add("microenvironment").add("scale");
  scale.attr("name", M.name);
  XNode& mesh = scale.add("mesh");
  mesh.attr("type", M.mesh.Cartesian_mesh ? "Cartesian" : "general");
  mesh.attr("uniform", bool_text(M.mesh.uniform_mesh));
  mesh.attr("regular", bool_text(M.mesh.regular_mesh));
  mesh.attr("units", M.mesh.units);
  {
    XNode& bb = mesh.add("bounding_box");
    bb.attr("type", "axis-aligned").attr("units", M.mesh.units);
    const std::vector<double>& b = M.mesh.bounding_box;
    bb.text = fmt("[%f %f %f %f %f %f]", b[0], b[1], b[2], b[3], b[4], b[5]);
  }
  if (M.mesh.Cartesian_mesh) {
    mesh.add("x_coordinates").attr("delimiter", ",").text = csv_of(M.mesh.x_coordinates, "%f");
    mesh.add("y_coordinates").attr("delimiter", ",").text = csv_of(M.mesh.y_coordinates, "%f");
    mesh.add("z_coordinates").attr("delimiter", ",").text = csv_of(M.mesh.z_coordinates, "%f");
  }
  XNode& vox = mesh.add("voxels");
  if (!save_mesh_as_matlab) {
    vox.attr("type", "xml");
    for (const Voxel& v : M.mesh.voxels) {
      XNode& x = vox.add("voxel");
      x.attr("ID", fmt("%d", v.mesh_index)).attr("type", "cube");
      x.add("center").attr("delimiter", ",").text =
          fmt("%f,%f,%f", v.center[0], v.center[1], v.center[2]);
      x.add("volume").text = fmt("%f", v.volume);
    }
  } else {
    vox.attr("type", "matlab");
    const std::string f = fmt("%s_mesh%d.mat", filename_base.c_str(), 0);
    M.mesh.write_to_matlab(f);
    vox.text = f;
  }
  XNode& dens = scale.add("densities");
  for (int j = 0; j < M.number_of_densities(); ++j) {
    XNode& d = dens.add("density");
    d.attr("name", M.density_names[j]).attr("units", M.density_units[j]);
    d.add("diffusion_constant").text = fmt("%f", M.diffusion_coefficients[j]);
    d.add("decay_rate").text = fmt("%f", M.decay_rates[j]);
  }
  XNode& data = scale.add("data");
  if (save_density_data_as_matlab) {
    const std::string f = fmt("%s_microenvironment%d.mat", filename_base.c_str(), 0);
    M.write_to_matlab(f);
    data.attr("type", "matlab");
    data.text = f;
  } else {
    data.attr("type", "xml");
    for (int j = 0; j < M.number_of_voxels(); ++j) {
      XNode& dv = data.add("density_vector");
      dv.attr("voxel_ID", fmt("%d", M.mesh.voxels[j].mesh_index)).attr("delimiter", ",");
      dv.text = csv_of(M.density_vector(j), "%.7e");
    }
  }
  g_doc = root;
  g_doc_built = true;
}

void update_document(const std::string& filename_base, Microenvironment& M) {
  XNode* md = g_doc.child("metadata");
  if (md) {
    if (XNode* t = md->child("current_time")) t->text = fmt("%f", default_metadata.current_time);
    if (XNode* t = md->child("current_runtime"))
      t->text = fmt("%f", default_metadata.current_runtime);
  }
  XNode* env = g_doc.child("microenvironment");
  XNode* scale = env ? env->child("scale") : nullptr;
  XNode* data = scale ? scale->child("data") : nullptr;
  if (!data) return;
  if (save_density_data_as_matlab) {
    const std::string f = fmt("%s_microenvironment%d.mat", filename_base.c_str(), 0);
    M.write_to_matlab(f);
    data->set("type", "matlab");
    if (data->kids.empty()) data->text = f;  // the text node, when there is one
  } else {
    data->set("type", "xml");
    // the existing density_vector entries, in order
    int j = 0;
    for (auto& k : data->kids) {
      if (k.name != "density_vector" || j >= M.number_of_voxels()) continue;
      k.text = csv_of(M.density_vector(j), "%.7e");
      ++j;
    }
  }
}

}  // namespace

void set_save_biovm_mesh_as_matlab(bool newvalue) { save_mesh_as_matlab = newvalue; }
void set_save_biovm_data_as_matlab(bool newvalue) { save_density_data_as_matlab = newvalue; }

void save_microenvironment_to_MultiCellDS_xml_pugi(std::string filename_base, Microenvironment& M) {
  // BioFVM_MultiCellDS.cpp:394-719
  std::cout << "Writing data to file " << filename_base << ".xml ... ";
  if (g_doc_built)
    update_document(filename_base, M);
  else
    build_document(filename_base, M);
  std::ofstream os(filename_base + ".xml");
  os << "<?xml version=\"1.0\"?>\n";
  write_node(os, g_doc, 0);
  std::cout << "done!" << std::endl;
}

void read_microenvironment_from_MultiCellDS_xml(Microenvironment& M, std::string filename) {
  // BioFVM_MultiCellDS.cpp:85-392
  std::cout << "Reading data from file " << filename << " ... ";
  std::ifstream in(filename);
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string text = ss.str();
  Parser parser(text);
  XNode doc;
  if (!parser.element(doc) || doc.name != "MultiCellDS") {
    std::cout << "could not parse " << filename << "!" << std::endl;
    return;
  }
  XNode* env = doc.child("microenvironment");
  if (!env) {
    std::cout << "done!" << std::endl;
    return;
  }
  for (XNode& scale : env->kids) {  // every microenvironment ("scale") in order
    M.name = scale.value("name");
    XNode* mesh = scale.child("mesh");
    if (!mesh) continue;
    const std::string type = mesh->value("type");
    const bool cartesian = (type == "Cartesian" || type == "cartesian");
    M.mesh.units = mesh->value("units");
    M.spatial_units = mesh->value("units");
    M.mesh.uniform_mesh = mesh->has("uniform") ? as_bool(mesh->value("uniform")) : true;
    M.mesh.regular_mesh = mesh->has("regular") ? as_bool(mesh->value("regular")) : true;
    XNode* bb = mesh->child("bounding_box");
    if (bb) csv_to_vector(bb->text.c_str(), M.mesh.bounding_box);
    if (cartesian) {
      std::vector<double>* coords[3] = {&M.mesh.x_coordinates, &M.mesh.y_coordinates,
                                        &M.mesh.z_coordinates};
      const char* names[3] = {"x_coordinates", "y_coordinates", "z_coordinates"};
      double d[3];
      for (int a = 0; a < 3; ++a) {
        XNode* c = mesh->child(names[a]);
        coords[a]->clear();
        if (c) csv_to_vector(c->text.c_str(), *coords[a]);
        d[a] = coords[a]->size() > 1 ? (*coords[a])[1] - (*coords[a])[0] : 1.0;
      }
      for (int a = 0; a < 3; ++a)
        if (coords[a]->size() < 2) d[a] = M.mesh.bounding_box[a + 3] - M.mesh.bounding_box[a];
      if (M.mesh.regular_mesh || M.mesh.uniform_mesh) {
        const std::vector<double> b = M.mesh.bounding_box;
        M.resize_space(b[0], b[3], b[1], b[4], b[2], b[5], d[0], d[1], d[2]);
      } else {
        std::cout << "Warning! BioFVM / MultiCellDS cannot currently fully initialize to "
                     "non-regular Cartesian data!"
                  << std::endl;
      }
    }
    if (!cartesian || !M.mesh.regular_mesh)
      std::cout << "Warning: voxel-list meshes (non-Cartesian or non-regular) are not read by "
                   "this library; the mesh is left as it is."
                << std::endl;

    XNode* dens = scale.child("densities");
    int index = -1;
    if (dens) {
      for (XNode& d : dens->kids) {
        if (d.name != "density") continue;
        if (index < 0)
          M.set_density(0, d.value("name"), d.value("units"));
        else
          M.add_density(d.value("name"), d.value("units"));
        ++index;
        if (XNode* x = d.child("diffusion_constant"))
          M.diffusion_coefficients[index] = std::strtod(x->text.c_str(), nullptr);
        if (XNode* x = d.child("decay_rate"))
          M.decay_rates[index] = std::strtod(x->text.c_str(), nullptr);
      }
    }
    XNode* data = scale.child("data");
    if (!data) continue;
    if (std::string(data->value("type")) == "matlab") {
      int rows = 0, columns = 0;
      FILE* fp = read_matlab_header(&rows, &columns, data->text);
      if (!fp) continue;
      const int start = rows > M.number_of_densities() ? 4 : 0;  // x, y, z, volume first
      std::vector<double> col(rows);
      for (int j = 0; j < columns && j < M.number_of_voxels(); ++j) {
        if (std::fread(col.data(), sizeof(double), rows, fp) != (size_t)rows) break;
        std::vector<double>& v = M.density_vector(j);
        for (int r = start; r < rows && r - start < (int)v.size(); ++r) v[r - start] = col[r];
      }
      std::fclose(fp);
    } else {
      int j = 0;
      for (XNode& k : data->kids) {
        if (k.name != "density_vector" || j >= M.number_of_voxels()) continue;
        csv_to_vector(k.text.c_str(), M.density_vector(j));
        ++j;
      }
    }
  }
  std::cout << "done!" << std::endl;
}

}  // namespace BioFVM
