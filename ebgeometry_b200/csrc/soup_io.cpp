// Mesh files -> triangle soup (host C++): the reading half of the reference's
// Parser::readIntoDCEL (ParserImplem.hpp:1752-1800) for STL, OBJ, PLY and legacy VTK, followed by
// its vertex merging (Soup::compress, SoupImplem.hpp:78-145).  The rules that decide which
// triangles a file yields follow the reference's readers:
//   STL  ASCII when the first 256 bytes contain "solid", a newline, "facet" and "normal" (in any
//        case), else binary (ParserImplem.hpp:59-90); ASCII reads the first solid only, one facet per
//        "facet" line and one vertex per "vertex" line (:186-250); binary reads the 50-byte records
//        and keeps the triangles of the smallest attribute id (:251-357);
//   OBJ  "v x y z" records and "f" records whose tokens start with a 1-based or negative vertex
//        index; faces of fewer than three vertices are dropped (:1661-1733);
//   PLY  ascii / binary_little_endian / binary_big_endian; the x, y, z scalar properties of the
//        vertex element and the list property of the face element (:374-890);
//   VTK  legacy ASCII POLYDATA: POINTS, then POLYGONS as count-prefixed lists or as OFFSETS /
//        CONNECTIVITY arrays (:906-1645).
// Vertex merging: the soup's positions are sorted lexicographically (x, then y, then z) and equal
// positions become one vertex; facets keep their order and their vertex count (a triangle mesh
// takes triangles only; a polygon mesh takes any face of three or more vertices).
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "capi_common.h"
#include "ebgeometry_b200.h"

struct ebg_soup
{
  std::vector<double>  v;   // 3 per vertex
  std::vector<int32_t> f;   // the faces' vertex indices, face after face
  std::vector<int64_t> off; // face k is f[off[k] .. off[k + 1])
  bool                 triangles = true;
};

namespace {

struct RawSoup
{
  std::vector<double>               v;
  std::vector<std::vector<int64_t>> f;
};

std::string lower(std::string s)
{
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return char(std::tolower(c)); });
  return s;
}

std::string extension(const std::string& path)
{
  const size_t dot = path.find_last_of('.');
  return dot == std::string::npos ? std::string() : lower(path.substr(dot + 1));
}

bool readAll(const std::string& path, std::string& data)
{
  std::ifstream is(path, std::ios::binary);
  if (!is) {
    return false;
  }
  std::ostringstream ss;
  ss << is.rdbuf();
  data = ss.str();
  return true;
}

// ---- STL ------------------------------------------------------------------------------------------
bool stlIsAscii(const std::string& data)
{
  const std::string head = lower(data.substr(0, std::min<size_t>(256, data.size())));
  return head.find("solid") != std::string::npos && head.find('\n') != std::string::npos &&
         head.find("facet") != std::string::npos && head.find("normal") != std::string::npos;
}

bool readStlAscii(const std::string& data, RawSoup& s, std::string& msg)
{
  std::istringstream in(data);
  std::string        line;
  bool               inSolid = false;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string        w;
    ls >> w;
    if (!inSolid) {
      inSolid = (w == "solid");
      continue;
    }
    if (w == "endsolid") {
      return true;
    }
    if (w == "facet") {
      s.f.emplace_back();
    }
    else if (w == "vertex") {
      if (s.f.empty()) {
        msg = "STL vertex outside a facet";
        return false;
      }
      double x = 0, y = 0, z = 0;
      ls >> x >> y >> z;
      s.v.insert(s.v.end(), {x, y, z});
      s.f.back().push_back(int64_t(s.v.size() / 3 - 1));
    }
  }
  if (!inSolid) {
    msg = "no 'solid' in the ASCII STL file";
    return false;
  }
  return true;
}

bool readStlBinary(const std::string& data, RawSoup& s, std::string& msg)
{
  if (data.size() < 84) {
    msg = "binary STL shorter than its header";
    return false;
  }
  uint32_t n = 0;
  std::memcpy(&n, data.data() + 80, 4);
  if (data.size() < 84 + size_t(n) * 50) {
    msg = "binary STL shorter than its triangle count";
    return false;
  }
  // the triangles of the smallest attribute id
  uint16_t keep = 0xffff;
  for (uint32_t i = 0; i < n; i++) {
    uint16_t id = 0;
    std::memcpy(&id, data.data() + 84 + size_t(i) * 50 + 48, 2);
    keep = std::min(keep, id);
  }
  for (uint32_t i = 0; i < n; i++) {
    const char* r  = data.data() + 84 + size_t(i) * 50;
    uint16_t    id = 0;
    std::memcpy(&id, r + 48, 2);
    if (id != keep) {
      continue;
    }
    std::vector<int64_t> facet;
    for (int c = 0; c < 3; c++) {
      float xyz[3];
      std::memcpy(xyz, r + 12 + 12 * c, 12);
      s.v.insert(s.v.end(), {double(xyz[0]), double(xyz[1]), double(xyz[2])});
      facet.push_back(int64_t(s.v.size() / 3 - 1));
    }
    s.f.push_back(facet);
  }
  return true;
}

// ---- OBJ ------------------------------------------------------------------------------------------
bool readObj(const std::string& data, RawSoup& s, std::string& msg)
{
  (void)msg;
  std::istringstream in(data);
  std::string        line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string        w;
    ls >> w;
    if (w == "v") {
      double x = 0, y = 0, z = 0;
      ls >> x >> y >> z;
      s.v.insert(s.v.end(), {x, y, z});
    }
    else if (w == "f") {
      std::vector<int64_t> facet;
      std::string          tok;
      while (ls >> tok) {
        const std::string head = tok.substr(0, tok.find('/'));
        char*             end  = nullptr;
        const long        idx  = std::strtol(head.c_str(), &end, 10);
        if (end == head.c_str()) {
          continue;
        }
        if (idx > 0) {
          facet.push_back(int64_t(idx) - 1);
        }
        else if (idx < 0) {
          facet.push_back(int64_t(s.v.size() / 3) + idx);
        }
      }
      if (facet.size() >= 3) {
        s.f.push_back(facet);
      }
    }
  }
  return true;
}

// ---- PLY ------------------------------------------------------------------------------------------
struct PlyProp
{
  std::string name, type;            // scalar: type; list: the index type
  bool        list = false;
  std::string countType;             // list only
};
struct PlyElement
{
  std::string          name;
  int64_t              count = 0;
  std::vector<PlyProp> props;
};

int plySize(const std::string& t)
{
  if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") {
    return 1;
  }
  if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") {
    return 2;
  }
  if (t == "int" || t == "uint" || t == "float" || t == "int32" || t == "uint32" || t == "float32") {
    return 4;
  }
  if (t == "double" || t == "float64") {
    return 8;
  }
  return 0;
}

// one binary scalar of PLY type t at p (byte order: big when swap is set) as a double
double plyValue(const char* p, const std::string& t, bool swap)
{
  const int n = plySize(t);
  char      b[8];
  for (int i = 0; i < n; i++) {
    b[i] = swap ? p[n - 1 - i] : p[i];
  }
  if (t == "char" || t == "int8") {
    return double(*reinterpret_cast<const int8_t*>(b));
  }
  if (t == "uchar" || t == "uint8") {
    return double(*reinterpret_cast<const uint8_t*>(b));
  }
  if (t == "short" || t == "int16") {
    int16_t x;
    std::memcpy(&x, b, 2);
    return double(x);
  }
  if (t == "ushort" || t == "uint16") {
    uint16_t x;
    std::memcpy(&x, b, 2);
    return double(x);
  }
  if (t == "int" || t == "int32") {
    int32_t x;
    std::memcpy(&x, b, 4);
    return double(x);
  }
  if (t == "uint" || t == "uint32") {
    uint32_t x;
    std::memcpy(&x, b, 4);
    return double(x);
  }
  if (t == "float" || t == "float32") {
    float x;
    std::memcpy(&x, b, 4);
    return double(x);
  }
  double x;
  std::memcpy(&x, b, 8);
  return x;
}

bool readPly(const std::string& data, RawSoup& s, std::string& msg)
{
  size_t pos = 0;
  auto   nextLine = [&](std::string& line) -> bool {
    if (pos >= data.size()) {
      return false;
    }
    const size_t e = data.find('\n', pos);
    line           = data.substr(pos, (e == std::string::npos ? data.size() : e) - pos);
    pos            = e == std::string::npos ? data.size() : e + 1;
    if (!line.empty() && line.back() == '\r') {
      line.pop_back();
    }
    return true;
  };
  std::string             line, format;
  std::vector<PlyElement> elems;
  if (!nextLine(line) || line.rfind("ply", 0) != 0) {
    msg = "not a PLY file";
    return false;
  }
  while (nextLine(line)) {
    std::istringstream ls(line);
    std::string        w;
    ls >> w;
    if (w == "format") {
      ls >> format;
    }
    else if (w == "element") {
      PlyElement e;
      ls >> e.name >> e.count;
      elems.push_back(e);
    }
    else if (w == "property" && !elems.empty()) {
      PlyProp p;
      std::string t;
      ls >> t;
      if (t == "list") {
        p.list = true;
        ls >> p.countType >> p.type >> p.name;
      }
      else {
        p.type = t;
        ls >> p.name;
      }
      elems.back().props.push_back(p);
    }
    else if (w == "end_header") {
      break;
    }
  }
  const bool ascii = format == "ascii";
  const bool swap  = format == "binary_big_endian";
  if (!ascii && format != "binary_little_endian" && !swap) {
    msg = "unknown PLY format '" + format + "'";
    return false;
  }
  for (const PlyElement& e : elems) {
    const bool isVertex = e.name == "vertex", isFace = e.name == "face";
    int        ix = -1, iy = -1, iz = -1;
    for (size_t k = 0; k < e.props.size(); k++) {
      ix = (e.props[k].name == "x") ? int(k) : ix;
      iy = (e.props[k].name == "y") ? int(k) : iy;
      iz = (e.props[k].name == "z") ? int(k) : iz;
    }
    for (int64_t r = 0; r < e.count; r++) {
      double               xyz[3] = {0, 0, 0};
      std::vector<int64_t> facet;
      bool                 gotList = false;
      std::istringstream   ls;
      if (ascii) {
        if (!nextLine(line)) {
          msg = "PLY data ends early";
          return false;
        }
        ls.str(line);
      }
      for (size_t k = 0; k < e.props.size(); k++) {
        const PlyProp& p = e.props[k];
        if (p.list) {
          double cnt = 0;
          if (ascii) {
            ls >> cnt;
          }
          else {
            const int sz = plySize(p.countType);
            if (sz == 0 || pos + size_t(sz) > data.size()) {
              msg = "PLY list count type or data size";
              return false;
            }
            cnt = plyValue(data.data() + pos, p.countType, swap);
            pos += size_t(sz);
          }
          std::vector<int64_t> idx(size_t(std::max(0.0, cnt)));
          for (auto& x : idx) {
            double val = 0;
            if (ascii) {
              ls >> val;
            }
            else {
              const int sz = plySize(p.type);
              if (sz == 0 || pos + size_t(sz) > data.size()) {
                msg = "PLY list index type or data size";
                return false;
              }
              val = plyValue(data.data() + pos, p.type, swap);
              pos += size_t(sz);
            }
            x = int64_t(val);
          }
          if (isFace && !gotList) {
            facet   = idx;
            gotList = true;
          }
        }
        else {
          double val = 0;
          if (ascii) {
            ls >> val;
          }
          else {
            const int sz = plySize(p.type);
            if (sz == 0 || pos + size_t(sz) > data.size()) {
              msg = "PLY property type or data size";
              return false;
            }
            val = plyValue(data.data() + pos, p.type, swap);
            pos += size_t(sz);
          }
          if (int(k) == ix) {
            xyz[0] = val;
          }
          else if (int(k) == iy) {
            xyz[1] = val;
          }
          else if (int(k) == iz) {
            xyz[2] = val;
          }
        }
      }
      if (isVertex) {
        s.v.insert(s.v.end(), {xyz[0], xyz[1], xyz[2]});
      }
      else if (isFace) {
        s.f.push_back(facet);
      }
    }
  }
  return true;
}

// ---- VTK (legacy ASCII POLYDATA) --------------------------------------------------------------------
bool readVtk(const std::string& data, RawSoup& s, std::string& msg)
{
  std::istringstream in(data);
  std::string        line;
  for (int i = 0; i < 3; i++) {
    if (!std::getline(in, line)) {
      msg = "VTK header ends early";
      return false;
    }
  }
  {
    std::istringstream ls(line);
    std::string        fmt;
    ls >> fmt;
    if (fmt != "ASCII") {
      msg = "only ASCII legacy VTK files are read";
      return false;
    }
  }
  std::string w;
  while (in >> w) {
    if (w == "POINTS") {
      int64_t     n = 0;
      std::string type;
      in >> n >> type;
      for (int64_t i = 0; i < n; i++) {
        double x = 0, y = 0, z = 0;
        in >> x >> y >> z;
        s.v.insert(s.v.end(), {x, y, z});
      }
    }
    else if (w == "POLYGONS") {
      int64_t n = 0, size = 0;
      in >> n >> size;
      std::string next;
      const auto  mark = in.tellg();
      in >> next;
      if (next == "OFFSETS") {
        std::string type;
        in >> type;
        std::vector<int64_t> off(size_t(std::max<int64_t>(n, 0)));
        for (auto& o : off) {
          in >> o;
        }
        std::string kw;
        while (in >> kw && kw != "CONNECTIVITY") {
        }
        if (kw != "CONNECTIVITY") {
          msg = "VTK OFFSETS without CONNECTIVITY";
          return false;
        }
        in >> type;
        std::vector<int64_t> conn(size_t(std::max<int64_t>(size, 0)));
        for (auto& c : conn) {
          in >> c;
        }
        for (int64_t i = 0; i + 1 < n; i++) {
          if (off[size_t(i)] < 0 || off[size_t(i + 1)] > int64_t(conn.size()) || off[size_t(i)] > off[size_t(i + 1)]) {
            msg = "VTK polygon offsets out of range";
            return false;
          }
          s.f.emplace_back(conn.begin() + off[size_t(i)], conn.begin() + off[size_t(i + 1)]);
        }
      }
      else {
        in.seekg(mark);
        for (int64_t i = 0; i < n; i++) {
          int64_t k = 0;
          in >> k;
          std::vector<int64_t> facet(size_t(std::max<int64_t>(k, 0)));
          for (auto& x : facet) {
            in >> x;
          }
          s.f.push_back(facet);
        }
      }
    }
  }
  return true;
}

// ---- merging (Soup::compress) ---------------------------------------------------------------------
bool compressSoup(const RawSoup& raw, ebg_soup& out, std::string& msg)
{
  const int64_t nv = int64_t(raw.v.size() / 3);
  std::vector<int64_t> order(static_cast<size_t>(nv));
  for (int64_t i = 0; i < nv; i++) {
    order[size_t(i)] = i;
  }
  const double* V = raw.v.data();
  std::sort(order.begin(), order.end(), [V](int64_t a, int64_t b) {
    for (int c = 0; c < 3; c++) {
      if (V[3 * a + c] != V[3 * b + c]) {
        return V[3 * a + c] < V[3 * b + c];
      }
    }
    return a < b;
  });
  std::vector<int64_t> remap(size_t(nv), -1);
  out.v.clear();
  for (int64_t k = 0; k < nv; k++) {
    const int64_t i   = order[size_t(k)];
    const bool    dup = k > 0 && V[3 * i] == V[3 * order[size_t(k - 1)]] &&
                     V[3 * i + 1] == V[3 * order[size_t(k - 1)] + 1] && V[3 * i + 2] == V[3 * order[size_t(k - 1)] + 2];
    if (!dup) {
      out.v.insert(out.v.end(), {V[3 * i], V[3 * i + 1], V[3 * i + 2]});
    }
    remap[size_t(i)] = int64_t(out.v.size() / 3 - 1);
  }
  if (out.v.size() / 3 > size_t(INT32_MAX)) {
    msg = "more than 2^31-1 vertices";
    return false;
  }
  out.f.clear();
  out.f.reserve(raw.f.size() * 3);
  out.off.assign(1, 0);
  out.triangles = true;
  for (size_t t = 0; t < raw.f.size(); t++) {
    const auto& facet = raw.f[t];
    if (facet.size() < 3) {
      msg = "face " + std::to_string(t) + " has fewer than three vertices";
      return false;
    }
    out.triangles = out.triangles && facet.size() == 3;
    for (int64_t i : facet) {
      if (i < 0 || i >= nv) {
        msg = "face " + std::to_string(t) + " references vertex " + std::to_string(i) + " of " + std::to_string(nv);
        return false;
      }
      out.f.push_back(int32_t(remap[size_t(i)]));
    }
    out.off.push_back(int64_t(out.f.size()));
  }
  return true;
}

} // namespace

extern "C" {

ebg_status ebg_soup_read(const char* path, ebg_soup** out)
{
  if (path == nullptr || out == nullptr) {
    return ebg::setError(EBG_ERR_INVALID, "null path or output handle");
  }
  *out = nullptr;
  std::string data;
  if (!readAll(path, data)) {
    return ebg::setError(EBG_ERR_NOT_FOUND, std::string("cannot open '") + path + "'");
  }
  const std::string ext = extension(path);
  RawSoup           raw;
  std::string       msg;
  bool              ok = false;
  if (ext == "stl") {
    ok = stlIsAscii(data) ? readStlAscii(data, raw, msg) : readStlBinary(data, raw, msg);
  }
  else if (ext == "obj") {
    ok = readObj(data, raw, msg);
  }
  else if (ext == "ply") {
    ok = readPly(data, raw, msg);
  }
  else if (ext == "vtk") {
    ok = readVtk(data, raw, msg);
  }
  else {
    return ebg::setError(EBG_ERR_INVALID, "unsupported file type '" + ext + "' (stl, obj, ply, vtk)");
  }
  if (!ok) {
    return ebg::setError(EBG_ERR_INVALID, std::string(path) + ": " + msg);
  }
  auto* s = new ebg_soup;
  if (!compressSoup(raw, *s, msg)) {
    delete s;
    return ebg::setError(EBG_ERR_INVALID, std::string(path) + ": " + msg);
  }
  *out = s;
  return EBG_OK;
}

ebg_status ebg_soup_sizes(const ebg_soup* s, int64_t* num_vertices, int64_t* num_triangles)
{
  if (s == nullptr || num_vertices == nullptr || num_triangles == nullptr) {
    return ebg::setError(EBG_ERR_INVALID, "null argument");
  }
  *num_vertices  = int64_t(s->v.size() / 3);
  *num_triangles = int64_t(s->off.size()) - 1;
  return EBG_OK;
}

ebg_status ebg_soup_copy(const ebg_soup* s, double* vertices, int32_t* triangles)
{
  if (s == nullptr || vertices == nullptr || triangles == nullptr) {
    return ebg::setError(EBG_ERR_INVALID, "null argument");
  }
  if (!s->triangles) {
    return ebg::setError(EBG_ERR_INVALID,
                         "the file has faces of more than three vertices: read it with ebg_soup_copy_polygons "
                         "(a triangle mesh takes triangles only)");
  }
  std::memcpy(vertices, s->v.data(), s->v.size() * sizeof(double));
  std::memcpy(triangles, s->f.data(), s->f.size() * sizeof(int32_t));
  return EBG_OK;
}

ebg_status ebg_soup_num_corners(const ebg_soup* s, int64_t* num_corners)
{
  if (s == nullptr || num_corners == nullptr) {
    return ebg::setError(EBG_ERR_INVALID, "null argument");
  }
  *num_corners = int64_t(s->f.size());
  return EBG_OK;
}

ebg_status ebg_soup_copy_polygons(const ebg_soup* s, double* vertices, int64_t* face_offsets, int32_t* face_vertices)
{
  if (s == nullptr || vertices == nullptr || face_offsets == nullptr || face_vertices == nullptr) {
    return ebg::setError(EBG_ERR_INVALID, "null argument");
  }
  std::memcpy(vertices, s->v.data(), s->v.size() * sizeof(double));
  std::memcpy(face_offsets, s->off.data(), s->off.size() * sizeof(int64_t));
  std::memcpy(face_vertices, s->f.data(), s->f.size() * sizeof(int32_t));
  return EBG_OK;
}

ebg_status ebg_soup_destroy(ebg_soup* s)
{
  delete s;
  return EBG_OK;
}

ebg_status ebg_mesh_create_from_file(const char* path, const ebg_build_opts* opts, ebg_mesh** out)
{
  ebg_soup*        s  = nullptr;
  const ebg_status rc = ebg_soup_read(path, &s);
  if (rc != EBG_OK) {
    return rc;
  }
  if (!s->triangles) {
    delete s;
    return ebg::setError(EBG_ERR_INVALID, std::string(path) +
                                              ": faces of more than three vertices (a triangle mesh takes triangles "
                                              "only; ebg_polymesh_create_from_file takes polygons)");
  }
  const ebg_status rc2 = ebg_mesh_create(s->v.data(), int64_t(s->v.size() / 3), s->f.data(), int64_t(s->f.size() / 3),
                                         opts, out);
  delete s;
  return rc2;
}

} // extern "C"
