// stage_loader.cpp — scene files: the `.stage` parser and scene builder, and the ASCII PLY
// reader for their meshes (pbrt_stage_* / pbrt_scene_load / pbrt_ply_read in
// include/pbrt_b200.h). Host code only.
//
// Follows the reference's loader:
//   tokens      src/loader/parser/lexer.rs:123-360 (keywords, signed decimal numbers, quoted
//               strings, `#` comments to the end of the line; any other character ends the
//               token stream)
//   grammar     src/loader/parser.rs:26-367
//   building    src/loader/visitors/scene_builder.rs: objects are popped from a stack, so the
//               scene and every compound list their members in reverse file order; a
//               transform block folds its steps as identity * step_n * ... * step_1 in f64
//               (Transform::mul, src/geom/transform.rs:119-127; the sequential 4x4 product of
//               src/geom/matrix4.rs:216-232); rotation inverses are transposes, translation
//               inverses negations (transform.rs:43-72)
//   lights      src/loader.rs:36-42 (a point light at (0, 2, 1) of intensity 15 and a
//               white-to-(0.5, 0.7, 1.0) background, added to every scene)
//   camera      src/loader/visitors/scene_builder.rs:62-91 with src/config.rs:112-129
//   PLY         src/loader/ply/ply_loader.rs:206-320, src/loader/mesh_loader.rs:13-85
// Transforms are composed in f64 as the reference composes them, then rounded to FP32 for
// the device.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pbrt_b200.h"

namespace {

struct StageError : std::runtime_error {
  int code;
  StageError(const std::string& m, int c = PBRT_ERR_INVALID_ARGUMENT) : std::runtime_error(m), code(c) {}
};

// ---- PLY ---------------------------------------------------------------------------------
enum class PlyType { I8, U8, I16, U16, I32, U32, F32, F64, Bad };

PlyType ply_type(const std::string& s) {  // ply_data_type.rs:17-37
  if (s == "char" || s == "int8") return PlyType::I8;
  if (s == "uchar" || s == "uint8") return PlyType::U8;
  if (s == "short" || s == "int16") return PlyType::I16;
  if (s == "ushort" || s == "uint16") return PlyType::U16;
  if (s == "int" || s == "int32") return PlyType::I32;
  if (s == "uint" || s == "uint32") return PlyType::U32;
  if (s == "float" || s == "float32") return PlyType::F32;
  if (s == "double" || s == "float64") return PlyType::F64;
  return PlyType::Bad;
}

struct PlyProp {
  std::string name;
  bool list = false;
  PlyType type = PlyType::Bad;  // the value type (list items)
};
struct PlyElement {
  std::string name;
  uint64_t count = 0;
  std::vector<PlyProp> props;
};

bool parse_int(const std::string& s, long long* v) {
  if (s.empty()) return false;
  char* end = nullptr;
  errno = 0;
  const long long x = std::strtoll(s.c_str(), &end, 10);
  if (errno || *end) return false;
  *v = x;
  return true;
}

std::vector<std::string> split_ws(const std::string& line) {
  std::vector<std::string> out;
  std::istringstream is(line);
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

// read_ply_data + MeshBuilder: x, y, z of every vertex (f32 text rounded as parse::<f32>),
// the index lists of every face (int or uint items), each reversed when `reverse`.
void read_ply(const std::string& path, bool reverse, std::vector<float>* verts, std::vector<uint32_t>* idx) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw StageError("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string data = ss.str();
  enum { kHeader, kFormat, kElement, kProperty, kData } state = kHeader;
  std::vector<PlyElement> elems;
  size_t cur = 0;
  uint64_t cur_count = 0;
  uint64_t vertex_count = 0;
  size_t pos = 0;
  uint64_t lineno = 0;
  while (pos <= data.size()) {
    size_t nl = data.find('\n', pos);
    if (nl == std::string::npos) nl = data.size();
    std::string line = data.substr(pos, nl - pos);
    pos = nl + 1;
    ++lineno;
    const std::vector<std::string> seg = split_ws(line);
    if (seg.empty() || seg[0].compare(0, 7, "comment") == 0) continue;
    const std::string where = path + ":" + std::to_string(lineno) + ": ";
    switch (state) {
      case kHeader:
        if (seg.size() != 1 || seg[0] != "ply") throw StageError(where + "a PLY file starts with 'ply'");
        state = kFormat;
        break;
      case kFormat:
        if (seg.size() != 3 || seg[0] != "format" || seg[1] != "ascii" || seg[2] != "1.0")
          throw StageError(where + "only 'format ascii 1.0' is read");
        state = kElement;
        break;
      case kProperty:
        if (seg[0] == "property") {
          PlyProp p;
          if (seg.size() == 3) {
            p.type = ply_type(seg[1]);
            p.name = seg[2];
          } else if (seg.size() == 5 && seg[1] == "list") {
            p.list = true;
            if (ply_type(seg[2]) == PlyType::Bad) throw StageError(where + "unknown PLY type " + seg[2]);
            p.type = ply_type(seg[3]);
            p.name = seg[4];
          } else {
            throw StageError(where + "malformed property");
          }
          if (p.type == PlyType::Bad) throw StageError(where + "unknown PLY type");
          elems.back().props.push_back(p);
          break;
        }
        state = kElement;
        [[fallthrough]];  // the line opens the next element or ends the header
      case kElement: {
        long long cnt = 0;
        if (seg.size() == 3 && seg[0] == "element" && (seg[1] == "vertex" || seg[1] == "face")) {
          if (!parse_int(seg[2], &cnt) || cnt < 0) throw StageError(where + "bad element count");
          elems.push_back(PlyElement{seg[1], uint64_t(cnt), {}});
          state = kProperty;
        } else if (seg.size() == 1 && seg[0] == "end_header") {
          state = kData;
          cur = 0;
          cur_count = 0;
          if (elems.empty()) throw StageError(where + "no element");
        } else {
          throw StageError(where + "expected 'element vertex', 'element face' or 'end_header'");
        }
        break;
      }
      case kData: {
        if (++cur_count > elems[cur].count) {  // ply_loader.rs:304-311
          ++cur;
          cur_count = 0;
          if (cur >= elems.size()) throw StageError(where + "more data lines than elements");
        }
        const PlyElement& e = elems[cur];
        size_t k = 0;
        float xyz[3] = {0, 0, 0};
        int have_xyz = 0;
        for (const PlyProp& p : e.props) {
          if (!p.list) {
            if (k >= seg.size()) throw StageError(where + "missing value");
            const std::string& v = seg[k++];
            if (e.name == "vertex" && (p.name == "x" || p.name == "y" || p.name == "z")) {
              const int a = p.name[0] - 'x';
              char* end = nullptr;
              if (p.type == PlyType::F32) {
                xyz[a] = std::strtof(v.c_str(), &end);
              } else if (p.type == PlyType::F64) {
                xyz[a] = float(std::strtod(v.c_str(), &end));
              } else {
                throw StageError(where + "vertex coordinates must be float or double");
              }
              if (!end || *end) throw StageError(where + "bad number " + v);
              have_xyz |= 1 << a;
            }
            continue;
          }
          long long n = 0;
          if (k >= seg.size() || !parse_int(seg[k], &n) || n < 0 || k + 1 + size_t(n) > seg.size())
            throw StageError(where + "bad list");
          ++k;
          const bool indices = e.name == "face" && (p.name == "vertex_index" || p.name == "vertex_indices") &&
                               (p.type == PlyType::I32 || p.type == PlyType::U32);
          if (indices) {
            if (n != 3) throw StageError(where + "faces must be triangles");
            uint32_t tri[3];
            for (int j = 0; j < 3; ++j) {
              long long x = 0;
              if (!parse_int(seg[k + j], &x) || x < 0 || x > 0xFFFFFFFFll) throw StageError(where + "bad index");
              tri[j] = uint32_t(x);
            }
            for (int j = 0; j < 3; ++j) idx->push_back(reverse ? tri[2 - j] : tri[j]);
          }
          k += size_t(n);
        }
        if (e.name == "vertex") {
          if (have_xyz != 7) throw StageError(where + "a vertex needs x, y and z");
          verts->insert(verts->end(), xyz, xyz + 3);
          ++vertex_count;
        }
        break;
      }
    }
  }
  if (state != kData) throw StageError(path + ": no end_header");
  for (uint32_t v : *idx)
    if (v >= vertex_count) throw StageError(path + ": a face names a missing vertex");
}

// ---- `.stage` tokens -----------------------------------------------------------------------
struct Tok {
  enum Kind { Kw, Id, Num, Str, Sym, End } kind = End;
  std::string s;
  double v = 0;
};

const char* const kKeywords[] = {
    "aabox", "camera", "reverse", "checkerboard", "color", "csg", "compound", "cylinder", "dielectric",
    "diffuse_light", "elem", "file", "focal_length", "intersection", "lambertian", "look", "metal", "mesh",
    "object", "pos", "pin_hole", "plane", "radius", "rectangle", "rotate_x", "rotate_y", "rotate_z", "scene",
    "simple", "sphere", "substraction", "thin_lens", "transform", "transformed", "translate", "union", "up"};

bool is_digit(char c) { return c >= '0' && c <= '9'; }
// Letters start identifiers; bytes of non-ASCII characters count as letters, so that such a
// character makes an (unknown) identifier, as Rust's char::is_alphabetic mostly would.
bool is_alpha(char c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || static_cast<unsigned char>(c) >= 0x80;
}

std::vector<Tok> tokenize(const std::string& t) {
  std::vector<Tok> out;
  size_t i = 0;
  const size_t n = t.size();
  for (;;) {
    while (i < n && std::isspace(static_cast<unsigned char>(t[i]))) ++i;
    if (i >= n) break;
    const char c = t[i];
    Tok k;
    if (c == '#') {
      while (i < n && t[i] != '\n') ++i;
      continue;
    }
    if (c == '{' || c == '}' || c == '[' || c == ']' || c == '(' || c == ')') {
      k.kind = Tok::Sym;
      k.s = std::string(1, c);
      ++i;
    } else if (c == '"') {
      size_t j = i + 1;
      while (j < n && t[j] != '"') ++j;
      if (j == i + 1) break;  // an empty string is no token (lexer.rs:205-222)
      k.kind = Tok::Str;
      k.s = t.substr(i + 1, j - i - 1);
      i = j + 1;
    } else if (is_digit(c) || c == '+' || c == '-') {
      // sign? digits+ ('.' digits*)?  (lexer.rs:224-293)
      size_t j = i;
      if (t[j] == '+' || t[j] == '-') ++j;
      const size_t d0 = j;
      while (j < n && is_digit(t[j])) ++j;
      if (j > d0 && j < n && t[j] == '.') {
        ++j;
        while (j < n && is_digit(t[j])) ++j;
      }
      const std::string num = t.substr(i, j - i);
      if (j == d0) throw StageError("bad number '" + num + "'");
      k.kind = Tok::Num;
      k.v = std::strtod(num.c_str(), nullptr);
      i = j;
    } else if (is_alpha(c)) {
      size_t j = i;
      while (j < n && (is_alpha(t[j]) || is_digit(t[j]) || t[j] == '_')) ++j;
      k.s = t.substr(i, j - i);
      k.kind = Tok::Id;
      for (const char* kw : kKeywords)
        if (k.s == kw) k.kind = Tok::Kw;
      i = j;
    } else {
      break;  // a character that starts no token ends the stream
    }
    out.push_back(k);
  }
  return out;
}

// ---- f64 transforms --------------------------------------------------------------------------
struct M4d {
  double m[4][4];
  static M4d identity() {
    M4d r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0;
    return r;
  }
  M4d operator*(const M4d& o) const {  // matrix4.rs:216-232
    M4d r{};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double acc = 0.0;
        for (int k = 0; k < 4; ++k) acc += m[i][k] * o.m[k][j];
        r.m[i][j] = acc;
      }
    return r;
  }
  M4d transposed() const {
    M4d r{};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) r.m[i][j] = m[j][i];
    return r;
  }
};
struct Xfd {
  M4d mat, inv;
  Xfd operator*(const Xfd& o) const { return Xfd{mat * o.mat, o.inv * inv}; }  // transform.rs:119-127
};
Xfd translation(double x, double y, double z) {
  Xfd t{M4d::identity(), M4d::identity()};
  t.mat.m[0][3] = x; t.mat.m[1][3] = y; t.mat.m[2][3] = z;
  t.inv.m[0][3] = -x; t.inv.m[1][3] = -y; t.inv.m[2][3] = -z;
  return t;
}
Xfd rotation(char axis, double a) {  // matrix4.rs:44-66
  const double s = std::sin(a), c = std::cos(a);
  M4d m = M4d::identity();
  if (axis == 'x') { m.m[1][1] = c; m.m[1][2] = -s; m.m[2][1] = s; m.m[2][2] = c; }
  else if (axis == 'y') { m.m[0][0] = c; m.m[0][2] = s; m.m[2][0] = -s; m.m[2][2] = c; }
  else { m.m[0][0] = c; m.m[0][1] = -s; m.m[1][0] = s; m.m[1][1] = c; }
  return Xfd{m, m.transposed()};
}
void rows(const M4d& m, float* out) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) out[4 * r + c] = float(m.m[r][c]);
}

}  // namespace

// ---- the stage -------------------------------------------------------------------------------
struct pbrt_stage {
  std::vector<pbrt_csg_elem_desc> csg;
  std::vector<std::vector<float>> mesh_v;
  std::vector<std::vector<uint32_t>> mesh_i;
  std::vector<pbrt_mesh_desc> meshes;
  std::vector<pbrt_material_desc> materials;
  std::vector<pbrt_object_desc> objects;
  std::vector<pbrt_node_desc> nodes;
  std::vector<uint32_t> children, roots;
  std::vector<pbrt_light_desc> lights;
  pbrt_camera_desc camera{};
  float lens[2] = {0.f, 0.f};
  uint32_t bvh_bins = 0, bvh_max_leaf = 0;
};

namespace {

class StageParser {
 public:
  StageParser(const std::string& text, const pbrt_stage_options& opt, pbrt_stage* st)
      : toks_(tokenize(text)), opt_(opt), st_(st) {}

  void run() {
    camera();
    expect_kw("scene");
    std::vector<uint32_t> top;
    while (i_ < toks_.size()) {
      expect_kw("object");
      top.push_back(object());
    }
    st_->roots.assign(top.rbegin(), top.rend());  // visit_scene pops: reverse order
    if (st_->roots.empty()) throw StageError("the scene holds no object");
    for (size_t k = 0; k < st_->meshes.size(); ++k) {
      st_->meshes[k].vertices = st_->mesh_v[k].data();
      st_->meshes[k].indices = st_->mesh_i[k].data();
    }
  }

 private:
  const Tok& next() {
    static const Tok end;
    return i_ < toks_.size() ? toks_[i_++] : end;
  }
  bool peek_kw(const char* w) const { return i_ < toks_.size() && toks_[i_].kind == Tok::Kw && toks_[i_].s == w; }
  void expect_kw(const char* w) {
    const Tok& t = next();
    if (t.kind != Tok::Kw || t.s != w) throw StageError(std::string("expected '") + w + "'");
  }
  void expect_sym(char c) {
    const Tok& t = next();
    if (t.kind != Tok::Sym || t.s[0] != c) throw StageError(std::string("expected '") + c + "'");
  }
  std::string kw() {
    const Tok& t = next();
    return t.kind == Tok::Kw ? t.s : std::string();
  }
  double number() {
    const Tok& t = next();
    if (t.kind != Tok::Num) throw StageError("expected a number");
    return t.v;
  }
  void vector(double* v) {
    for (int a = 0; a < 3; ++a) v[a] = number();
  }

  // parser.rs:34-83 + scene_builder.rs:62-91 (fov, near, far, resolution from the options)
  void camera() {
    expect_kw("camera");
    const std::string k = kw();
    if (k != "pin_hole" && k != "thin_lens") throw StageError("unknown camera type");
    double pos[3], look[3], up[3];
    expect_kw("pos");
    vector(pos);
    expect_kw("look");
    vector(look);
    expect_kw("up");
    vector(up);
    pbrt_camera_desc& c = st_->camera;
    if (k == "thin_lens") {  // visit_camera_thin_lens: the file's radius and focal length
      expect_kw("radius");
      st_->lens[0] = float(number());
      expect_kw("focal_length");
      st_->lens[1] = float(number());
      c.thin_lens = 1;
      c.lens_radius = st_->lens[0];
      c.focal_distance = st_->lens[1];
    }
    c.width = opt_.width ? opt_.width : 800;
    c.height = opt_.height ? opt_.height : 600;
    const double fov_deg = opt_.fov_deg != 0.0 ? opt_.fov_deg : 90.0;
    c.fov = float(fov_deg * 3.141592653589793 / 180.0);
    c.near = float(opt_.near != 0.0 ? opt_.near : 0.0001);
    c.far = float(opt_.far != 0.0 ? opt_.far : 1000.0);
    for (int a = 0; a < 3; ++a) {
      c.position[a] = float(pos[a]);
      c.look_at[a] = float(look[a]);
      c.up[a] = float(up[a]);
    }
  }

  uint32_t add_node(const pbrt_node_desc& n) {
    if (st_->nodes.size() >= 0x7FFFFFFFu) throw StageError("too many objects");
    st_->nodes.push_back(n);
    return uint32_t(st_->nodes.size() - 1);
  }

  // parser.rs:104-139, scene_builder.rs:95-116
  uint32_t object() {
    const std::string k = kw();
    pbrt_node_desc n{};
    if (k == "simple") {
      pbrt_object_desc o{};
      shape(&o);
      pbrt_material_desc m{};
      material(&m);
      st_->materials.push_back(m);
      o.material = uint32_t(st_->materials.size() - 1);
      st_->objects.push_back(o);
      n.kind = PBRT_NODE_SIMPLE;
      n.object = uint32_t(st_->objects.size() - 1);
      return add_node(n);
    }
    if (k == "transformed") {
      expect_kw("object");
      const uint32_t child = object();
      const Xfd x = transform();
      n.kind = PBRT_NODE_TRANSFORMED;
      n.first = uint32_t(st_->children.size());
      n.count = 1;
      st_->children.push_back(child);
      rows(x.mat, n.to_world);
      rows(x.inv, n.to_local);
      return add_node(n);
    }
    if (k == "compound") {
      expect_sym('{');
      std::vector<uint32_t> kids;
      for (;;) {
        const Tok& t = next();
        if (t.kind == Tok::Kw && t.s == "object") kids.push_back(object());
        else if (t.kind == Tok::Sym && t.s == "}") break;
        else throw StageError("expected } or object");
      }
      n.kind = PBRT_NODE_COMPOUND;
      n.first = uint32_t(st_->children.size());
      n.count = uint32_t(kids.size());
      st_->children.insert(st_->children.end(), kids.rbegin(), kids.rend());  // popped: reverse order
      return add_node(n);
    }
    throw StageError("expected simple, transformed or compound");
  }

  void shape(pbrt_object_desc* o) {
    const std::string k = kw();
    if (k == "aabox") {
      double e[3];
      vector(e);
      o->shape = PBRT_SHAPE_AABOX;
      for (int a = 0; a < 3; ++a) o->extent[a] = float(e[a]);
    } else if (k == "sphere") {
      o->shape = PBRT_SHAPE_SPHERE;
      o->radius = float(number());
    } else if (k == "cylinder") {
      o->shape = PBRT_SHAPE_CYLINDER;
      o->radius = float(number());
      o->height = float(number());
    } else if (k == "rectangle") {  // the two numbers are Rectangle::new's width and height
      o->shape = PBRT_SHAPE_RECTANGLE;
      o->radius = float(number());
      o->height = float(number());
    } else if (k == "plane") {
      o->shape = PBRT_SHAPE_PLANE;
    } else if (k == "mesh") {
      expect_kw("file");
      const Tok& f = next();
      if (f.kind != Tok::Str) throw StageError("expected a mesh file name");
      bool rev = false;
      if (peek_kw("reverse")) {
        ++i_;
        rev = true;
      }
      o->shape = PBRT_SHAPE_MESH;
      o->mesh = mesh(f.s, rev);
    } else if (k == "csg") {  // parser.rs:157-196, scene_builder.rs:118-143
      const std::string op = kw();
      o->shape = PBRT_SHAPE_CSG;
      if (op == "union") o->csg_op = PBRT_CSG_UNION;
      else if (op == "intersection") o->csg_op = PBRT_CSG_INTERSECTION;
      else if (op == "substraction") o->csg_op = PBRT_CSG_SUBTRACTION;
      else throw StageError("expected intersection, union or subtraction");
      expect_sym('{');
      std::vector<pbrt_csg_elem_desc> elems;
      for (;;) {
        const Tok& t = next();
        if (t.kind == Tok::Kw && t.s == "elem") {
          pbrt_object_desc e{};
          shape(&e);
          if (e.shape == PBRT_SHAPE_CSG)
            throw StageError("a constructive solid nested in another is not supported", PBRT_ERR_UNSUPPORTED);
          const Xfd x = transform();
          pbrt_csg_elem_desc d{};
          d.shape = e.shape;
          d.mesh = e.mesh;
          d.radius = e.radius;
          d.height = e.height;
          for (int a = 0; a < 3; ++a) d.extent[a] = e.extent[a];
          rows(x.mat, d.to_world);
          rows(x.inv, d.to_local);
          elems.push_back(d);
        } else if (t.kind == Tok::Sym && t.s == "}") {
          break;
        } else {
          throw StageError("expected } or elem");
        }
      }
      o->csg_first = uint32_t(st_->csg.size());
      o->csg_count = uint32_t(elems.size());
      st_->csg.insert(st_->csg.end(), elems.rbegin(), elems.rend());  // popped: reverse order
    } else {
      throw StageError("expected a shape");
    }
  }

  uint32_t mesh(const std::string& name, bool rev) {
    const auto key = std::make_pair(name, rev);
    auto it = mesh_ids_.find(key);
    if (it != mesh_ids_.end()) return it->second;
    std::string path = name;
    if (opt_.base_dir && opt_.base_dir[0] && !name.empty() && name[0] != '/')
      path = std::string(opt_.base_dir) + "/" + name;
    std::vector<float> v;
    std::vector<uint32_t> ix;
    read_ply(path, rev, &v, &ix);
    pbrt_mesh_desc md{};
    md.vertex_count = uint32_t(v.size() / 3);
    md.triangle_count = uint32_t(ix.size() / 3);
    st_->mesh_v.push_back(std::move(v));
    st_->mesh_i.push_back(std::move(ix));
    st_->meshes.push_back(md);
    const uint32_t id = uint32_t(st_->meshes.size() - 1);
    mesh_ids_[key] = id;
    return id;
  }

  void material(pbrt_material_desc* m) {  // parser.rs:249-283
    const std::string k = kw();
    if (k == "dielectric") {
      m->kind = PBRT_MAT_DIELECTRIC;
      m->ior = float(number());
    } else if (k == "metal") {
      m->kind = PBRT_MAT_METAL;
      m->fuzz = float(number());
    } else if (k == "lambertian") {
      m->kind = PBRT_MAT_LAMBERTIAN;
    } else if (k == "diffuse_light") {
      m->kind = PBRT_MAT_DIFFUSE_LIGHT;
    } else {
      throw StageError("expected lambertian, dielectric, metal");
    }
    const std::string t = kw();
    double c[3];
    if (t == "color") {
      vector(c);
      m->texture = PBRT_TEXTURE_COLOR;
      for (int a = 0; a < 3; ++a) m->color[a] = float(c[a]);
    } else if (t == "checkerboard") {
      double c2[3];
      vector(c);
      vector(c2);
      m->texture = PBRT_TEXTURE_CHECKERBOARD;
      for (int a = 0; a < 3; ++a) {
        m->color[a] = float(c[a]);
        m->color2[a] = float(c2[a]);
      }
      m->scale = float(number());
    } else {
      throw StageError("expected color, checkerboard");
    }
  }

  Xfd transform() {  // parser.rs:297-334, scene_builder.rs:200-212
    expect_kw("transform");
    expect_sym('{');
    std::vector<Xfd> steps;
    for (;;) {
      const Tok& t = next();
      if (t.kind == Tok::Kw && t.s == "translate") {
        double v[3];
        vector(v);
        steps.push_back(translation(v[0], v[1], v[2]));
      } else if (t.kind == Tok::Kw && (t.s == "rotate_x" || t.s == "rotate_y" || t.s == "rotate_z")) {
        steps.push_back(rotation(t.s.back(), number()));
      } else if (t.kind == Tok::Sym && t.s == "}") {
        break;
      } else {
        throw StageError("expected a transform step");
      }
    }
    Xfd r{M4d::identity(), M4d::identity()};
    for (auto it = steps.rbegin(); it != steps.rend(); ++it) r = r * *it;
    return r;
  }

  std::vector<Tok> toks_;
  size_t i_ = 0;
  const pbrt_stage_options& opt_;
  pbrt_stage* st_;
  std::map<std::pair<std::string, bool>, uint32_t> mesh_ids_;
};

void set_err(char* err, size_t len, const std::string& m) {
  if (err && len) {
    std::strncpy(err, m.c_str(), len - 1);
    err[len - 1] = '\0';
  }
}

}  // namespace

extern "C" {

int pbrt_stage_parse(const char* text, const pbrt_stage_options* options, pbrt_stage** out, char* err,
                     size_t err_len) {
  set_err(err, err_len, "");
  if (!text || !out) {
    set_err(err, err_len, "text or out is NULL");
    return PBRT_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  const pbrt_stage_options opt = options ? *options : pbrt_stage_options{};
  std::unique_ptr<pbrt_stage> st(new pbrt_stage);
  try {
    StageParser(text, opt, st.get()).run();
  } catch (const StageError& e) {
    set_err(err, err_len, e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_err(err, err_len, "out of host memory");
    return PBRT_ERR_OUT_OF_MEMORY;
  }
  if (!opt.no_loader_lights) {  // loader.rs:36-42
    pbrt_light_desc p{};
    p.kind = PBRT_LIGHT_POINT;
    p.position[1] = 2.0f;
    p.position[2] = 1.0f;
    for (int c = 0; c < 3; ++c) p.radiance[c] = 15.0f;
    pbrt_light_desc b{};
    b.kind = PBRT_LIGHT_BACKGROUND_INFINITE;
    for (int c = 0; c < 3; ++c) b.bottom[c] = 1.0f;
    b.top[0] = 0.5f;
    b.top[1] = 0.7f;
    b.top[2] = 1.0f;
    st->lights.push_back(p);
    st->lights.push_back(b);
  }
  st->bvh_bins = opt.bvh_bins;
  st->bvh_max_leaf = opt.bvh_max_leaf;
  *out = st.release();
  return PBRT_OK;
}

int pbrt_stage_describe(const pbrt_stage* st, pbrt_scene_desc* d, pbrt_camera_desc* camera, float* camera_lens) {
  if (!st) return PBRT_ERR_INVALID_ARGUMENT;
  if (d) {
    *d = pbrt_scene_desc{};
    d->meshes = st->meshes.data();
    d->mesh_count = uint32_t(st->meshes.size());
    d->materials = st->materials.data();
    d->material_count = uint32_t(st->materials.size());
    d->objects = st->objects.data();
    d->object_count = uint32_t(st->objects.size());
    d->lights = st->lights.data();
    d->light_count = uint32_t(st->lights.size());
    d->bvh_bins = st->bvh_bins;
    d->bvh_max_leaf = st->bvh_max_leaf;
    d->nodes = st->nodes.data();
    d->node_count = uint32_t(st->nodes.size());
    d->node_children = st->children.data();
    d->child_count = uint32_t(st->children.size());
    d->roots = st->roots.data();
    d->root_count = uint32_t(st->roots.size());
    d->csg_elems = st->csg.data();
    d->csg_elem_count = uint32_t(st->csg.size());
  }
  if (camera) *camera = st->camera;
  if (camera_lens) {
    camera_lens[0] = st->lens[0];
    camera_lens[1] = st->lens[1];
  }
  return PBRT_OK;
}

void pbrt_stage_destroy(pbrt_stage* st) { delete st; }

int pbrt_ply_read(const char* path, int reverse, float** vertices, uint32_t* vertex_count, uint32_t** indices,
                  uint32_t* triangle_count, char* err, size_t err_len) {
  set_err(err, err_len, "");
  if (!path || !vertices || !vertex_count || !indices || !triangle_count) return PBRT_ERR_INVALID_ARGUMENT;
  *vertices = nullptr;
  *indices = nullptr;
  std::vector<float> v;
  std::vector<uint32_t> ix;
  try {
    read_ply(path, reverse != 0, &v, &ix);
  } catch (const StageError& e) {
    set_err(err, err_len, e.what());
    return e.code;
  }
  float* pv = static_cast<float*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(float)));
  uint32_t* pi = static_cast<uint32_t*>(std::malloc(std::max<size_t>(1, ix.size()) * sizeof(uint32_t)));
  if (!pv || !pi) {
    std::free(pv);
    std::free(pi);
    return PBRT_ERR_OUT_OF_MEMORY;
  }
  if (!v.empty()) std::memcpy(pv, v.data(), v.size() * sizeof(float));
  if (!ix.empty()) std::memcpy(pi, ix.data(), ix.size() * sizeof(uint32_t));
  *vertices = pv;
  *indices = pi;
  *vertex_count = uint32_t(v.size() / 3);
  *triangle_count = uint32_t(ix.size() / 3);
  return PBRT_OK;
}

void pbrt_free(void* p) { std::free(p); }

}  // extern "C"
