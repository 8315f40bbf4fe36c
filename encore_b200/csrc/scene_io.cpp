// Scene front-end: PLY meshes and the reference's text scene files.
//
// Restates, in the reference's float operation order:
//   Model::loadPLY           ENCORE/src/scene/Model.cpp:396-482
//   Model::centerModel       ENCORE/src/scene/Model.cpp:109-141
//   Model::getCenterMatrix   ENCORE/src/scene/Model.cpp:143-173
//   Model::rotate            ENCORE/src/scene/Model.cpp:175-202
//   Scene::load              ENCORE/src/scene/Scene.cpp:184-209
//   Scene::HandleSceneVariable ENCORE/src/scene/Scene.cpp:78-183
//   RectangleLight geometry  ENCORE/src/scene/RectangleLight.cpp (constructor, Init)
//
// Differences, all on inputs the reference mishandles:
//   * the PLY header is parsed property by property, so x/y/z are found by
//     name (the reference takes the first three numbers of a vertex line) and
//     binary files are read too; faces keep the reference's rule of using
//     the first three indices of each face;
//   * an index out of range, a short file or a non-numeric token where a
//     number belongs is an error (the reference reads past its buffers or
//     loops);
//   * at end of file the reference runs the last command once more on the
//     failed stream (Scene.cpp:196-206); that repeat is not reproduced.
#include <cctype>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.h"
#include "scene.h"

namespace enc {
namespace {

struct Mesh {
  std::vector<float> v;         // 3 floats per vertex
  std::vector<uint32_t> f;      // 3 indices per face
};

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::ostringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

enum PType { T_I8, T_U8, T_I16, T_U16, T_I32, T_U32, T_F32, T_F64 };

PType ptype(const std::string& s) {
  if (s == "char" || s == "int8") return T_I8;
  if (s == "uchar" || s == "uint8") return T_U8;
  if (s == "short" || s == "int16") return T_I16;
  if (s == "ushort" || s == "uint16") return T_U16;
  if (s == "int" || s == "int32") return T_I32;
  if (s == "uint" || s == "uint32") return T_U32;
  if (s == "float" || s == "float32") return T_F32;
  if (s == "double" || s == "float64") return T_F64;
  throw std::runtime_error("PLY: unknown property type '" + s + "'");
}

int psize(PType t) {
  static const int sz[] = {1, 1, 2, 2, 4, 4, 4, 8};
  return sz[t];
}

struct Prop {
  std::string name;
  bool list = false;
  PType count_type = T_U8, type = T_F32;
};

struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Prop> props;
};

// Binary reader with the file's byte order.
struct BinCursor {
  const unsigned char* p;
  const unsigned char* end;
  bool big;
  double get(PType t) {
    const int n = psize(t);
    if (end - p < n) throw std::runtime_error("PLY: file ends inside the data");
    unsigned char b[8];
    for (int i = 0; i < n; ++i) b[i] = big ? p[n - 1 - i] : p[i];
    p += n;
    switch (t) {
      case T_I8: return (double)(int8_t)b[0];
      case T_U8: return (double)b[0];
      case T_I16: { int16_t x; std::memcpy(&x, b, 2); return x; }
      case T_U16: { uint16_t x; std::memcpy(&x, b, 2); return x; }
      case T_I32: { int32_t x; std::memcpy(&x, b, 4); return x; }
      case T_U32: { uint32_t x; std::memcpy(&x, b, 4); return x; }
      case T_F32: { float x; std::memcpy(&x, b, 4); return x; }
      default: { double x; std::memcpy(&x, b, 8); return x; }
    }
  }
};

// Whitespace-separated tokens of the ascii body.
struct TextCursor {
  const char* p;
  const char* end;
  const char* next() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
    if (p >= end) throw std::runtime_error("PLY: file ends inside the data");
    const char* s = p;
    while (p < end && !(*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
    return s;
  }
  // atof / atoi on the token, as the reference converts (Model.cpp:450-452, 471-473)
  double number() {
    const char* s = next();
    std::string tok(s, (size_t)(p - s));
    char* e = nullptr;
    const double x = std::strtod(tok.c_str(), &e);
    if (e == tok.c_str()) throw std::runtime_error("PLY: '" + tok + "' is not a number");
    return x;
  }
};

Mesh load_ply_mesh(const std::string& path) {
  const std::string buf = read_file(path);
  if (buf.compare(0, 3, "ply") != 0) throw std::runtime_error(path + " is not a PLY file");
  const size_t hend = buf.find("end_header");
  if (hend == std::string::npos) throw std::runtime_error("PLY: no end_header");
  size_t body = buf.find('\n', hend);
  body = body == std::string::npos ? buf.size() : body + 1;

  std::istringstream hs(buf.substr(0, hend));
  std::string line, format = "ascii";
  std::vector<Element> els;
  while (std::getline(hs, line)) {
    std::istringstream ls(line);
    std::string kw;
    ls >> kw;
    if (kw == "format") {
      ls >> format;
    } else if (kw == "element") {
      Element e;
      ls >> e.name >> e.count;
      els.push_back(e);
    } else if (kw == "property") {
      if (els.empty()) throw std::runtime_error("PLY: property before element");
      Prop pr;
      std::string t;
      ls >> t;
      if (t == "list") {
        std::string ct, it;
        ls >> ct >> it;
        pr.list = true;
        pr.count_type = ptype(ct);
        pr.type = ptype(it);
      } else {
        pr.type = ptype(t);
      }
      ls >> pr.name;
      els.back().props.push_back(pr);
    }
  }
  if (format != "ascii" && format != "binary_little_endian" && format != "binary_big_endian")
    throw std::runtime_error("PLY: unknown format " + format);
  const bool ascii = format == "ascii";

  Mesh m;
  bool have_v = false, have_f = false;
  TextCursor tc{buf.data() + body, buf.data() + buf.size()};
  BinCursor bc{(const unsigned char*)buf.data() + body,
               (const unsigned char*)buf.data() + buf.size(), format == "binary_big_endian"};
  auto get = [&](PType t) { return ascii ? tc.number() : bc.get(t); };
  for (const Element& e : els) {
    const bool is_v = e.name == "vertex" && !have_v;
    const bool is_f = e.name == "face" && !have_f;
    int ix = -1, iy = -1, iz = -1, ilist = -1;
    for (size_t k = 0; k < e.props.size(); ++k) {
      const Prop& pr = e.props[k];
      if (is_v && !pr.list) {
        if (pr.name == "x") ix = (int)k;
        if (pr.name == "y") iy = (int)k;
        if (pr.name == "z") iz = (int)k;
      }
      if (is_f && pr.list && ilist < 0) ilist = (int)k;
    }
    if (is_v && (ix < 0 || iy < 0 || iz < 0)) throw std::runtime_error("PLY: vertex without x/y/z");
    if (is_f && ilist < 0) throw std::runtime_error("PLY: face without an index list");
    if (e.count > buf.size() - body) throw std::runtime_error("PLY: element count beyond the file size");
    if (is_v) m.v.resize(3 * e.count);
    if (is_f) m.f.reserve(3 * e.count);
    for (uint64_t i = 0; i < e.count; ++i) {
      for (size_t k = 0; k < e.props.size(); ++k) {
        const Prop& pr = e.props[k];
        if (!pr.list) {
          const double x = get(pr.type);
          if (is_v) {
            if ((int)k == ix) m.v[3 * i + 0] = (float)x;
            if ((int)k == iy) m.v[3 * i + 1] = (float)x;
            if ((int)k == iz) m.v[3 * i + 2] = (float)x;
          }
          continue;
        }
        const double cnt = get(pr.count_type);
        if (!(cnt >= 0) || cnt > 1e6) throw std::runtime_error("PLY: bad list length");
        const uint32_t n = (uint32_t)cnt;
        if (is_f && (int)k == ilist && n < 3) throw std::runtime_error("PLY: face with fewer than 3 vertices");
        for (uint32_t j = 0; j < n; ++j) {
          const double x = get(pr.type);
          if (is_f && (int)k == ilist && j < 3) {
            if (!(x >= 0)) throw std::runtime_error("PLY: negative vertex index");
            m.f.push_back((uint32_t)x);
          }
        }
      }
    }
    have_v |= is_v;
    have_f |= is_f;
  }
  if (!have_v) throw std::runtime_error("PLY: no vertex element");
  const size_t nv = m.v.size() / 3;
  for (uint32_t idx : m.f)
    if (idx >= nv) throw std::runtime_error("PLY: vertex index out of range");
  return m;
}

// Model::rotate (Model.cpp:175-202): identity for |angle| under 1e-7 rad,
// else the axis-angle matrix (the axis is used as given, not normalised).
void rotation(float angle, const float u[3], float R[16]) {
  for (int i = 0; i < 16; ++i) R[i] = (i % 5 == 0) ? 1.f : 0.f;
  const float rad = (float)(angle / 180.0 * M_PI);
  if (rad <= 0.0000001 && rad >= -0.0000001) return;
  const float c = std::cos(rad);
  const float s = std::sin(rad);
  const float k = 1 - c;
  R[0] = c + k * u[0] * u[0];
  R[4] = k * u[1] * u[0] - s * u[2];
  R[8] = k * u[2] * u[0] + s * u[1];
  R[1] = k * u[0] * u[1] + s * u[2];
  R[5] = c + k * u[1] * u[1];
  R[9] = k * u[2] * u[1] - s * u[0];
  R[2] = k * u[0] * u[2] - s * u[1];
  R[6] = k * u[1] * u[2] + s * u[0];
  R[10] = c + k * u[2] * u[2];
}

// Model::centerModel + getCenterMatrix: scale the model so its longest side
// is `size`, move its box centre to `center`, rotate (Model.cpp:109-173).
void center_model(std::vector<float>& v, const enc_model_xform& xf) {
  const size_t nv = v.size() / 3;
  // loadPLY starts its running bounds at POS_INF = FLT_MAX and NEG_INF =
  // FLT_MIN (Common.h:28-29, Model.cpp:62-63), the smallest positive float:
  // a model lying entirely at or below zero on an axis gets FLT_MIN as its
  // maximum there, which shifts its centre.  Reproduced for identical output.
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
  for (size_t i = 0; i < nv; ++i)
    for (int a = 0; a < 3; ++a) {
      const float x = v[3 * i + a];
      hi[a] = hi[a] > x ? hi[a] : x;  // max()/min() as loadPLY tracks them
      lo[a] = lo[a] < x ? lo[a] : x;
    }
  float len[3];
  for (int a = 0; a < 3; ++a) len[a] = hi[a] - lo[a];
  const float longest = len[0] > (len[1] > len[2] ? len[1] : len[2]) ? len[0]
                                                                       : (len[1] > len[2] ? len[1] : len[2]);
  const float scale = xf.size / longest;
  float off[3];
  for (int a = 0; a < 3; ++a) {
    const float mid = (hi[a] + lo[a]) * 0.5f;
    off[a] = mid * scale - xf.center[a];
  }
  float m[16];
  rotation(xf.angle_deg, xf.axis, m);
  m[12] = -off[0] * m[0] - off[1] * m[4] - off[2] * m[8];
  m[13] = -off[0] * m[1] - off[1] * m[5] - off[2] * m[9];
  m[14] = -off[0] * m[2] - off[1] * m[6] - off[2] * m[10];
  for (int i : {0, 1, 2, 4, 5, 6, 8, 9, 10}) m[i] *= scale;
  for (size_t i = 0; i < nv; ++i) {
    const float x = v[3 * i], y = v[3 * i + 1], z = v[3 * i + 2];
    v[3 * i + 0] = x * m[0] + y * m[4] + z * m[8] + m[12];
    v[3 * i + 1] = x * m[1] + y * m[5] + z * m[9] + m[13];
    v[3 * i + 2] = x * m[2] + y * m[6] + z * m[10] + m[14];
  }
}

// Appends a loaded, centred PLY model's triangles (Triangle(v0, v1, v2) per
// face, Model.cpp:475-478) to the scene in face order.
uint32_t append_ply(enc_scene_s* s, const std::string& path, const enc_model_xform& xf,
                    int32_t material) {
  Mesh m = load_ply_mesh(path);
  center_model(m.v, xf);
  const uint32_t nf = (uint32_t)(m.f.size() / 3);
  const int32_t prim0 = (int32_t)s->desc.nprims;
  s->verts.reserve(s->verts.size() + 9 * (size_t)nf);
  for (uint32_t t = 0; t < nf; ++t) {
    for (int k = 0; k < 3; ++k) {
      const float* p = &m.v[3 * (size_t)m.f[3 * t + k]];
      s->verts.insert(s->verts.end(), p, p + 3);
    }
    s->prim_of_tri.push_back(prim0 + (int32_t)t);
    s->material_of_tri.push_back(material);
  }
  s->ntris += nf;
  s->desc.nprims += nf;
  s->desc.ntris = s->ntris;
  s->desc.nmodels += 1;
  return nf;
}

// The ceiling light of RectangleLight::RectangleLight: a 30 x 30 square at
// y = 49.99999 facing down, split as (v0, v1, v2), (v2, v3, v0).
void append_rect_light(enc_scene_s* s, const float color[3], int32_t material) {
  const float y = 49.99999f;
  const float q[4][3] = {{15, y, 15}, {-15, y, 15}, {-15, y, -15}, {15, y, -15}};
  const int tri[2][3] = {{0, 1, 2}, {2, 3, 0}};
  const int32_t prim = (int32_t)s->desc.nprims;
  for (auto& t : tri) {
    for (int k = 0; k < 3; ++k) s->verts.insert(s->verts.end(), q[t[k]], q[t[k]] + 3);
    s->prim_of_tri.push_back(prim);
    s->material_of_tri.push_back(material);
  }
  s->ntris += 2;
  s->desc.ntris = s->ntris;
  s->desc.nprims += 1;
  s->desc.nmodels += 1;
  enc_scene_light L{};
  L.kind = ENC_LIGHT_RECT;
  for (int a = 0; a < 3; ++a) {
    L.center[a] = (q[0][a] + q[1][a] + q[2][a] + q[3][a]) / 4.0f;
    L.color[a] = color[a];
  }
  L.size = 30.f;
  s->lights.push_back(L);
}

// Scene::load's token stream: whitespace-separated words, '*' starts a
// comment running to the end of its line.
struct SceneTokens {
  std::string text;
  size_t pos = 0;
  int line = 1;
  bool word(std::string* out) {
    for (;;) {
      while (pos < text.size() && std::isspace((unsigned char)text[pos])) {
        if (text[pos] == '\n') ++line;
        ++pos;
      }
      if (pos >= text.size()) return false;
      const size_t b = pos;
      while (pos < text.size() && !std::isspace((unsigned char)text[pos])) ++pos;
      *out = text.substr(b, pos - b);
      if ((*out)[0] != '*') return true;
      while (pos < text.size() && text[pos] != '\n') ++pos;  // file.getline
    }
  }
  std::string need_word(const char* what) {
    std::string w;
    if (!word(&w)) throw std::runtime_error(std::string("scene file ends inside ") + what);
    return w;
  }
  float number(const char* what) {
    const std::string w = need_word(what);
    char* e = nullptr;
    const float x = std::strtof(w.c_str(), &e);  // operator>>(float&)
    if (e == w.c_str())
      throw std::runtime_error("line " + std::to_string(line) + ": '" + w + "' is not a number in " + what);
    return x;
  }
};

void load_scene_file(enc_scene_s* s, const std::string& path, const char* model_dir) {
  SceneTokens tk;
  tk.text = read_file(path);
  int32_t material = -1;
  std::string var;
  auto resolve = [&](const std::string& f) {
    if (!model_dir || !*model_dir || (!f.empty() && f[0] == '/')) return f;
    return std::string(model_dir) + "/" + f;
  };
  while (tk.word(&var)) {
    if (var == "BACKGROUND_COLOR") {
      for (int i = 0; i < 4; ++i) s->desc.background[i] = tk.number("BACKGROUND_COLOR");
    } else if (var == "POINT_LIGHT") {
      enc_scene_light L{};
      L.kind = ENC_LIGHT_POINT;
      for (int a = 0; a < 3; ++a) L.center[a] = tk.number("POINT_LIGHT");
      for (int a = 0; a < 3; ++a) L.color[a] = tk.number("POINT_LIGHT");
      s->lights.insert(s->lights.begin(), L);  // m_pLightList.push_front
    } else if (var == "RECT_LIGHT") {
      float c[3];
      for (int a = 0; a < 3; ++a) c[a] = tk.number("RECT_LIGHT");
      append_rect_light(s, c, material);
    } else if (var == "MATERIAL") {
      std::array<float, 13> mt;
      for (float& x : mt) x = tk.number("MATERIAL");
      s->materials.push_back(mt);
      material = (int32_t)s->materials.size() - 1;
    } else if (var == "SPHERE") {
      for (int i = 0; i < 9; ++i) tk.number("SPHERE");
      s->desc.nprims += 1;  // a SpherePrim: one primitive, no triangles
      s->desc.nmodels += 1;
      s->desc.nspheres += 1;
    } else if (var == "CAMERA") {
      float c[13];
      for (float& x : c) x = tk.number("CAMERA");
      for (int a = 0; a < 3; ++a) {
        s->desc.cam_eye[a] = c[a];
        s->desc.cam_look[a] = c[3 + a];
        s->desc.cam_up[a] = c[6 + a];
      }
      s->desc.cam_fov_deg = c[9];
      s->desc.cam_aspect = c[10];
      s->desc.cam_near = c[11];
      s->desc.cam_far = c[12];
      s->desc.has_camera = 1;
    } else if (var == "MODEL") {
      const std::string f = tk.need_word("MODEL");
      enc_model_xform xf;
      for (int a = 0; a < 3; ++a) xf.center[a] = tk.number("MODEL");
      xf.size = tk.number("MODEL");
      xf.angle_deg = tk.number("MODEL");
      for (int a = 0; a < 3; ++a) xf.axis[a] = tk.number("MODEL");
      const size_t dot = f.find_last_of('.');
      const std::string ext = dot == std::string::npos ? "" : f.substr(dot + 1);
      if (ext != "ply" && ext != "PLY")
        throw std::runtime_error("MODEL " + f + ": only PLY meshes are supported");
      append_ply(s, resolve(f), xf, material);
    } else {
      s->desc.nunknown += 1;  // the reference prints a warning and reads on
    }
  }
  s->desc.nmaterials = (uint32_t)s->materials.size();
  s->desc.nlights = (uint32_t)s->lights.size();
}

}  // namespace
}  // namespace enc

using namespace enc;

extern "C" {

enc_status enc_scene_load_ply(const char* path, const enc_model_xform* xform, enc_scene* out) {
  if (!path || !xform || !out) {
    set_error("enc_scene_load_ply: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  enc_scene s = new (std::nothrow) enc_scene_s();
  if (!s) return ENC_ERR_OUT_OF_MEMORY;
  try {
    append_ply(s, path, *xform, -1);
  } catch (const std::bad_alloc&) {
    delete s;
    set_error("enc_scene_load_ply: host out of memory");
    return ENC_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& ex) {
    delete s;
    set_error(std::string("enc_scene_load_ply: ") + ex.what());
    return ENC_ERR_INVALID_ARG;
  }
  *out = s;
  return ENC_OK;
}

enc_status enc_scene_load_file(const char* path, const char* model_dir, enc_scene* out) {
  if (!path || !out) {
    set_error("enc_scene_load_file: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *out = nullptr;
  enc_scene s = new (std::nothrow) enc_scene_s();
  if (!s) return ENC_ERR_OUT_OF_MEMORY;
  try {
    load_scene_file(s, path, model_dir);
  } catch (const std::bad_alloc&) {
    delete s;
    set_error("enc_scene_load_file: host out of memory");
    return ENC_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& ex) {
    delete s;
    set_error(std::string("enc_scene_load_file: ") + ex.what());
    return ENC_ERR_INVALID_ARG;
  }
  *out = s;
  return ENC_OK;
}

enc_status enc_scene_desc_get(enc_scene scene, enc_scene_desc* desc) {
  if (!scene || !desc) {
    set_error("enc_scene_desc_get: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  *desc = scene->desc;
  desc->ntris = scene->ntris;
  return ENC_OK;
}

enc_status enc_scene_tris(enc_scene scene, float* tri_verts, uint32_t cap, uint32_t* ntris) {
  if (!scene || (!tri_verts && cap)) {
    set_error("enc_scene_tris: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const uint32_t n = cap < scene->ntris ? cap : scene->ntris;
  if (n) std::memcpy(tri_verts, scene->verts.data(), 9 * sizeof(float) * (size_t)n);
  if (ntris) *ntris = scene->ntris;
  return ENC_OK;
}

enc_status enc_scene_prims(enc_scene scene, int32_t* prim_of_tri, int32_t* material_of_tri,
                           uint32_t cap) {
  if (!scene) {
    set_error("enc_scene_prims: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const uint32_t n = cap < scene->ntris ? cap : scene->ntris;
  const bool loaded = scene->prim_of_tri.size() == scene->ntris;
  for (uint32_t i = 0; i < n; ++i) {
    if (prim_of_tri) prim_of_tri[i] = loaded ? scene->prim_of_tri[i] : (int32_t)i;
    if (material_of_tri) material_of_tri[i] = loaded ? scene->material_of_tri[i] : -1;
  }
  return ENC_OK;
}

enc_status enc_scene_materials(enc_scene scene, float* out13, uint32_t cap, uint32_t* n) {
  if (!scene || (!out13 && cap)) {
    set_error("enc_scene_materials: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const uint32_t m = (uint32_t)scene->materials.size();
  for (uint32_t i = 0; i < m && i < cap; ++i)
    std::memcpy(out13 + 13 * (size_t)i, scene->materials[i].data(), 13 * sizeof(float));
  if (n) *n = m;
  return ENC_OK;
}

enc_status enc_scene_lights(enc_scene scene, enc_scene_light* out, uint32_t cap, uint32_t* n) {
  if (!scene || (!out && cap)) {
    set_error("enc_scene_lights: null argument");
    return ENC_ERR_INVALID_ARG;
  }
  const uint32_t m = (uint32_t)scene->lights.size();
  for (uint32_t i = 0; i < m && i < cap; ++i) out[i] = scene->lights[i];
  if (n) *n = m;
  return ENC_OK;
}

}  // extern "C"
