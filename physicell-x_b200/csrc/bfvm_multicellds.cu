// bfvm_multicellds.cu -- the microenvironment's MultiCellDS output.
//
// Reference: add_BioFVM_substrates_to_open_xml_pugi (BioFVM/BioFVM_MultiCellDS.cpp:
// 518-823, its first call in a process, with the default
// save_mesh_as_matlab and save_density_data_as_matlab) puts a <domain>
// element under <microenvironment>: the Cartesian mesh (bounding box, the
// voxel-centre coordinates of each axis as "%f" text, the mesh file name),
// one <variable> per substrate (name, units, ID, diffusion coefficient and
// decay rate as "%f") and the density file name; it writes
// <base>_mesh0.mat (General_Mesh::write_to_matlab) and
// <base>_microenvironment0.mat (Microenvironment::write_to_matlab).
// save_BioFVM_to_MultiCellDS_xml_pugi (:1880-1890) saves the document with
// pugixml's default format.
//
// bfvm_write_multicellds writes the two MATLAB files from the device (the
// columns assembled there) and the document as it stands after that call --
// the MultiCellDS root with empty <metadata> and <cellular_information>
// (the reference fills those with the run's metadata, wall-clock
// timestamps included, and its agents) -- byte for byte as the reference
// saves it.  Text follows pugixml's default output: a declaration line, tab
// indentation, elements without children closed as "<name />", an element
// whose only child is text printed on one line; &, <, > escaped everywhere,
// and in attributes also " and the control characters other than tab.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bfvm_ctx.h"

namespace bfvm {
int write_matlab_columns(bfvm_ctx* c, const char* path, const char* name, bool densities, double x_start,
                         double y_start, double z_start);
}

namespace {

std::string escape(const char* s, bool attribute) {
  std::string o;
  for (const char* p = s; *p; ++p) {
    const char ch = *p;
    switch (ch) {
      case '&': o += "&amp;"; break;
      case '<': o += "&lt;"; break;
      case '>': o += "&gt;"; break;
      case '"':
        if (attribute)
          o += "&quot;";
        else
          o += ch;
        break;
      default:
        // control characters as numeric references: in attributes all but
        // tab, in text all but tab, line feed and carriage return
        if (static_cast<unsigned char>(ch) < 32 && ch != '\t' && (attribute || (ch != '\n' && ch != '\r'))) {
          o += "&#" + std::to_string(static_cast<int>(ch)) + ";";
        } else {
          o += ch;
        }
    }
  }
  return o;
}

struct Node {
  std::string name;
  std::vector<std::pair<std::string, std::string>> attrs;  // escaped on output
  std::string text;                                        // pcdata, when there are no children
  std::vector<Node> kids;
  Node& attr(const char* k, const std::string& v) {
    attrs.emplace_back(k, v);
    return *this;
  }
  Node& add(const char* n) {
    kids.push_back(Node{n, {}, {}, {}});
    return kids.back();
  }
};

void emit(const Node& n, int depth, std::string& out) {
  out.append(depth, '\t');
  out += '<';
  out += n.name;
  for (const auto& a : n.attrs) {
    out += ' ';
    out += a.first;
    out += "=\"";
    out += escape(a.second.c_str(), true);
    out += '"';
  }
  if (n.kids.empty() && n.text.empty()) {
    out += " />\n";
    return;
  }
  if (n.kids.empty()) {
    out += '>';
    out += escape(n.text.c_str(), false);
    out += "</";
    out += n.name;
    out += ">\n";
    return;
  }
  out += ">\n";
  for (const Node& k : n.kids) emit(k, depth + 1, out);
  out.append(depth, '\t');
  out += "</";
  out += n.name;
  out += ">\n";
}

std::string fmt_f(double v) {
  char b[512];
  std::snprintf(b, sizeof b, "%f", v);
  return b;
}

// Voxel centres of one axis as the reference's mesh holds them, start +
// (i + 0.5)*dx evaluated as one fused multiply-add, joined with spaces.
std::string coordinates(int n, double start, double dx) {
  std::string s;
  for (int i = 0; i < n; ++i) {
    if (i) s += ' ';
    s += fmt_f(std::fma(static_cast<double>(i) + 0.5, dx, start));
  }
  return s;
}

const char* base_name(const std::string& path) {
  const char* p = std::strrchr(path.c_str(), '/');
  return p ? p + 1 : path.c_str();
}

}  // namespace

extern "C" int bfvm_write_multicellds(bfvm_ctx* c, const char* filename_base, const char* domain_name,
                                      const char* mesh_units, const char* spatial_units, const char* time_units,
                                      const char* const* density_names, const char* const* density_units,
                                      const double* bounding_box, char* xml, size_t xml_capacity,
                                      size_t* xml_length) {
  if (!c || !filename_base || !domain_name || !mesh_units || !spatial_units || !time_units || !density_names ||
      !density_units || !bounding_box)
    return BFVM_ERR_ARG;
  for (int s = 0; s < c->S; ++s)
    if (!density_names[s] || !density_units[s]) return BFVM_ERR_ARG;
  const std::string base(filename_base);
  const std::string mesh_file = base + "_mesh0.mat";
  const std::string data_file = base + "_microenvironment0.mat";

  Node root{"MultiCellDS", {}, {}, {}};
  root.attr("version", "0.5").attr("type", "snapshot/simulation");
  root.add("metadata");
  Node& dom = root.add("microenvironment").add("domain");
  dom.attr("name", domain_name);
  Node& mesh = dom.add("mesh");
  mesh.attr("type", "Cartesian").attr("uniform", "true").attr("regular", "true").attr("units", mesh_units);
  {
    Node& bb = mesh.add("bounding_box");
    bb.attr("type", "axis-aligned").attr("units", mesh_units);
    std::string t;
    for (int q = 0; q < 6; ++q) {
      if (q) t += ' ';
      t += fmt_f(bounding_box[q]);
    }
    bb.text = t;
  }
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  const char* axis_names[3] = {"x_coordinates", "y_coordinates", "z_coordinates"};
  for (int a = 0; a < 3; ++a) {
    Node& co = mesh.add(axis_names[a]);
    co.text = coordinates(n_axis[a], bounding_box[a], c->dx);
    co.attr("delimiter", " ");
  }
  {
    Node& vox = mesh.add("voxels");
    vox.attr("type", "matlab");
    vox.add("filename").text = base_name(mesh_file);
  }
  Node& vars = dom.add("variables");
  for (int s = 0; s < c->S; ++s) {
    Node& v = vars.add("variable");
    v.attr("name", density_names[s]).attr("units", density_units[s]).attr("ID", std::to_string(s));
    Node& ps = v.add("physical_parameter_set");
    ps.add("conditions");
    Node& dc = ps.add("diffusion_coefficient");
    dc.text = fmt_f(c->D[s]);
    dc.attr("units", std::string(spatial_units) + "^2/" + time_units);
    Node& dr = ps.add("decay_rate");
    dr.text = fmt_f(c->decay[s]);
    dr.attr("units", std::string("1/") + time_units);
  }
  {
    Node& data = dom.add("data");
    data.attr("type", "matlab");
    data.add("filename").text = base_name(data_file);
  }
  root.add("cellular_information");

  std::string doc = "<?xml version=\"1.0\"?>\n";
  emit(root, 0, doc);

  int rc = bfvm::write_matlab_columns(c, mesh_file.c_str(), "mesh", false, bounding_box[0], bounding_box[1],
                                      bounding_box[2]);
  if (rc != BFVM_OK) return rc;
  rc = bfvm::write_matlab_columns(c, data_file.c_str(), "multiscale_microenvironment", true, bounding_box[0],
                                  bounding_box[1], bounding_box[2]);
  if (rc != BFVM_OK) return rc;
  const std::string xml_file = base + ".xml";
  FILE* fp = std::fopen(xml_file.c_str(), "wb");
  if (!fp) {
    std::fprintf(stderr, "biofvm_b200: cannot open %s for writing\n", xml_file.c_str());
    return BFVM_ERR_ARG;
  }
  const bool ok = std::fwrite(doc.data(), 1, doc.size(), fp) == doc.size();
  if (std::fclose(fp) != 0 || !ok) return BFVM_ERR_ARG;
  if (xml_length) *xml_length = doc.size();
  if (xml) {
    if (xml_capacity < doc.size() + 1) return BFVM_ERR_ARG;
    std::memcpy(xml, doc.c_str(), doc.size() + 1);
  }
  return BFVM_OK;
}
