// Gmsh 2.2 ASCII reader: triangles, and physical tags of boundary lines as
// face tags.  Replaces PETSc's DMPlexCreateGmsh (src/solvers/apsolver.cc:318-327)
// and the "Face Sets" handling of wxNodalDGgeometry2D::FacePair2d
// (src/lib/wxnodaldggeometry2d.cc:334-356).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "apollo_dg.h"

struct apollo_dg_mesh {
  std::vector<double> vx, vy;
  std::vector<int> etov, tag;
};

namespace {

unsigned long long edge_key(int a, int b) {
  return ((unsigned long long)(unsigned)std::min(a, b) << 32) | (unsigned)std::max(a, b);
}

// Nodes per element for the element types of a 2D mesh (Gmsh 2.2 numbering).
int nodes_of(int type) {
  switch (type) {
    case 1: return 2;   // line
    case 2: return 3;   // triangle
    case 3: return 4;   // quadrangle
    case 8: return 3;   // second-order line
    case 9: return 6;   // second-order triangle
    case 15: return 1;  // point
    default: return -1;
  }
}

std::string parse(std::istream& in, apollo_dg_mesh& m) {
  std::string line;
  bool have_format = false, have_nodes = false, have_elems = false;
  std::unordered_map<long long, int> node_index;
  std::vector<std::array<long long, 3>> tris;
  std::unordered_map<unsigned long long, int> line_tag;  // physical tag by edge (vertex indices)
  std::vector<std::pair<std::array<long long, 2>, int>> lines;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    if (line == "$MeshFormat") {
      std::getline(in, line);
      std::istringstream ss(line);
      double version;
      int file_type, data_size;
      if (!(ss >> version >> file_type >> data_size)) return "bad $MeshFormat line";
      if (version < 2.0 || version >= 3.0) return "only Gmsh 2.x meshes are read";
      if (file_type != 0) return "binary Gmsh files are not read (save as ASCII)";
      have_format = true;
    } else if (line == "$Nodes") {
      long long n;
      if (!(in >> n) || n < 3) return "bad node count";
      m.vx.resize(n);
      m.vy.resize(n);
      for (long long i = 0; i < n; ++i) {
        long long id;
        double x, y, z;
        if (!(in >> id >> x >> y >> z)) return "truncated $Nodes";
        node_index[id] = (int)i;
        m.vx[i] = x;
        m.vy[i] = y;
      }
      have_nodes = true;
    } else if (line == "$Elements") {
      long long n;
      if (!(in >> n) || n < 1) return "bad element count";
      for (long long i = 0; i < n; ++i) {
        long long id;
        int type, ntags;
        if (!(in >> id >> type >> ntags) || ntags < 0) return "truncated $Elements";
        std::vector<long long> tags(ntags);
        for (auto& t : tags)
          if (!(in >> t)) return "truncated element tags";
        const int nn = nodes_of(type);
        if (nn < 0) return "unsupported element type " + std::to_string(type);
        if (type == 3 || type == 8 || type == 9) return "only straight-sided triangles are supported";
        std::vector<long long> v(nn);
        for (auto& x : v)
          if (!(in >> x)) return "truncated element nodes";
        if (type == 2) tris.push_back({v[0], v[1], v[2]});
        if (type == 1) lines.push_back({{v[0], v[1]}, ntags > 0 ? (int)tags[0] : 0});
      }
      have_elems = true;
    } else if (line[0] == '$' && line.rfind("$End", 0) != 0) {
      // an unused section ($PhysicalNames, $Periodic, $NodeData, ...): skip to its end
      const std::string end = "$End" + line.substr(1);
      bool closed = false;
      while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line == end) {
          closed = true;
          break;
        }
      }
      if (!closed) return "unterminated section " + end.substr(4);
    }
  }
  if (!have_format || !have_nodes || !have_elems) return "missing $MeshFormat, $Nodes or $Elements";
  if (tris.empty()) return "no triangles";
  auto idx = [&](long long id, int* out) {
    auto it = node_index.find(id);
    if (it == node_index.end()) return false;
    *out = it->second;
    return true;
  };
  const int K = (int)tris.size();
  m.etov.resize((size_t)K * 3);
  for (int k = 0; k < K; ++k) {
    int a, b, c;
    if (!idx(tris[k][0], &a) || !idx(tris[k][1], &b) || !idx(tris[k][2], &c)) return "element references an unknown node";
    // counter-clockwise, as the reference-element map needs J > 0
    const double area2 = (m.vx[b] - m.vx[a]) * (m.vy[c] - m.vy[a]) - (m.vx[c] - m.vx[a]) * (m.vy[b] - m.vy[a]);
    if (area2 == 0.0) return "degenerate triangle " + std::to_string(k);
    if (area2 < 0) std::swap(b, c);
    m.etov[3 * k] = a;
    m.etov[3 * k + 1] = b;
    m.etov[3 * k + 2] = c;
  }
  for (auto& l : lines) {
    int a, b;
    if (!idx(l.first[0], &a) || !idx(l.first[1], &b)) return "line references an unknown node";
    if (l.second > 0) line_tag[edge_key(a, b)] = l.second;
  }
  // face tags.  Apollo first writes -label over every connectivity entry of an
  // element with a labelled face ("Face Sets"), then overwrites the interior
  // pairs; unlabelled boundary faces keep -1, i.e. boundary condition 1.  So
  // every unpaired face of an element takes its label.  Where an element's
  // faces carry different labels Apollo keeps the one DMPlex visits last (an
  // order PETSc defines); here each labelled unpaired face keeps its own
  // label and an unlabelled one takes the element's last labelled face's
  // (face order v0v1, v1v2, v2v0).
  static const int vn[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  std::unordered_map<unsigned long long, int> uses;
  uses.reserve((size_t)K * 2);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) ++uses[edge_key(m.etov[3 * k + vn[f][0]], m.etov[3 * k + vn[f][1]])];
  m.tag.assign((size_t)K * 3, 0);
  for (int k = 0; k < K; ++k) {
    int lab[3], last = 0;
    for (int f = 0; f < 3; ++f) {
      auto it = line_tag.find(edge_key(m.etov[3 * k + vn[f][0]], m.etov[3 * k + vn[f][1]]));
      lab[f] = it == line_tag.end() ? 0 : it->second;
      if (lab[f]) last = lab[f];
    }
    for (int f = 0; f < 3; ++f) {
      const unsigned long long e = edge_key(m.etov[3 * k + vn[f][0]], m.etov[3 * k + vn[f][1]]);
      if (uses[e] >= 2) continue;  // interior: paired, whatever its label
      m.tag[3 * k + f] = lab[f] ? lab[f] : (last ? last : 1);
    }
  }
  return "";
}

}  // namespace

extern "C" {

apollo_status apollo_dg_mesh_read_gmsh(const char* path, apollo_dg_mesh** out, char* err, int err_len) {
  if (!path || !out) return APOLLO_ERR_ARG;
  *out = nullptr;
  std::ifstream in(path);
  std::string e;
  apollo_dg_mesh* m = new apollo_dg_mesh();
  if (!in) e = std::string("cannot open ") + path;
  else e = parse(in, *m);
  if (!e.empty()) {
    delete m;
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.c_str());
    return APOLLO_ERR_MESH;
  }
  *out = m;
  return APOLLO_OK;
}

apollo_status apollo_dg_mesh_info(const apollo_dg_mesh* m, int* nverts, int* K) {
  if (!m) return APOLLO_ERR_ARG;
  if (nverts) *nverts = (int)m->vx.size();
  if (K) *K = (int)(m->etov.size() / 3);
  return APOLLO_OK;
}

apollo_status apollo_dg_mesh_arrays(const apollo_dg_mesh* m, double* vx, double* vy, int* etov, int* face_tag) {
  if (!m) return APOLLO_ERR_ARG;
  if (vx) std::copy(m->vx.begin(), m->vx.end(), vx);
  if (vy) std::copy(m->vy.begin(), m->vy.end(), vy);
  if (etov) std::copy(m->etov.begin(), m->etov.end(), etov);
  if (face_tag) std::copy(m->tag.begin(), m->tag.end(), face_tag);
  return APOLLO_OK;
}

apollo_status apollo_dg_mesh_destroy(apollo_dg_mesh* m) {
  delete m;
  return APOLLO_OK;
}

}  // extern "C"
