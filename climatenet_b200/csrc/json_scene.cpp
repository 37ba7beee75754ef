// json_scene.cpp — the reference's scene / parameter JSON and OBJ input.
//
// Keeps the key spellings the reference code actually reads
// (src/scene_building.cpp:49-202, 279-318; src/simulation_building.cpp:37-78)
// and rapidjson's typing rules: a value required as a double must be written
// as a floating-point literal ("1.0", "1e3"), an unsigned value as an integer.
// OBJ coordinates are rounded through float like tinyobj's real_t
// (src/geometry/io.cpp:65-121).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pdf.h"

namespace pdfb {
void set_global_error(const std::string& msg);  // api.cu
}

namespace {

struct LoadError {
  void operator=(const std::string& m) { pdfb::set_global_error(m); }
  void operator=(const char* m) { pdfb::set_global_error(m); }
} g_load_error;

// ---------------------------------------------------------------- JSON
struct JVal {
  enum Kind { Null, Bool, Int, Double, String, Array, Object } kind = Null;
  bool b = false;
  long long i = 0;
  double d = 0;
  std::string s;
  std::vector<JVal> a;
  std::vector<std::pair<std::string, JVal>> o;

  bool is_double() const { return kind == Double; }
  bool is_uint() const { return kind == Int && i >= 0 && i <= 0xffffffffLL; }
  bool is_number() const { return kind == Int || kind == Double; }
  double num() const { return kind == Int ? (double)i : d; }
  const JVal* find(const char* key) const {
    for (auto& kv : o)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

struct JParser {
  const char* p;
  const char* end;
  explicit JParser(const std::string& s) : p(s.data()), end(s.data() + s.size()) {}
  [[noreturn]] void error(const char* what) {
    const char* stop = (end - p > 24) ? p + 24 : end;
    throw std::invalid_argument(std::string("JSON parse error: ") + what + " at \"" + std::string(p, stop) + "\"");
  }
  void ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  JVal parse() {
    ws();
    JVal v = value();
    ws();
    if (p != end) error("trailing characters");
    return v;
  }
  JVal value() {
    ws();
    if (p >= end) error("unexpected end");
    JVal v;
    if (*p == '{') {
      v.kind = JVal::Object;
      ++p;
      ws();
      if (p < end && *p == '}') {
        ++p;
        return v;
      }
      while (true) {
        ws();
        if (p >= end || *p != '"') error("expected key");
        std::string k = str();
        ws();
        if (p >= end || *p != ':') error("expected ':'");
        ++p;
        v.o.push_back({k, value()});
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == '}') {
          ++p;
          break;
        }
        error("expected ',' or '}'");
      }
    } else if (*p == '[') {
      v.kind = JVal::Array;
      ++p;
      ws();
      if (p < end && *p == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.a.push_back(value());
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == ']') {
          ++p;
          break;
        }
        error("expected ',' or ']'");
      }
    } else if (*p == '"') {
      v.kind = JVal::String;
      v.s = str();
    } else if (!strncmp(p, "true", std::min<size_t>(4, end - p)) && end - p >= 4) {
      v.kind = JVal::Bool;
      v.b = true;
      p += 4;
    } else if (!strncmp(p, "false", std::min<size_t>(5, end - p)) && end - p >= 5) {
      v.kind = JVal::Bool;
      p += 5;
    } else if (!strncmp(p, "null", std::min<size_t>(4, end - p)) && end - p >= 4) {
      p += 4;
    } else {
      const char* s = p;
      bool is_float = false;
      if (p < end && *p == '-') ++p;
      if (p >= end || !(*p >= '0' && *p <= '9')) error("invalid value");
      while (p < end && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' || *p == '+' || *p == '-')) {
        if (*p == '.' || *p == 'e' || *p == 'E') is_float = true;
        ++p;
      }
      std::string t(s, p);
      char* e = nullptr;
      if (is_float) {
        v.kind = JVal::Double;
        v.d = std::strtod(t.c_str(), &e);
      } else {
        v.kind = JVal::Int;
        v.i = std::strtoll(t.c_str(), &e, 10);
      }
      if (!e || *e) error("invalid number");
    }
    return v;
  }
  std::string str() {
    ++p;
    std::string out;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) error("bad escape");
        switch (*p) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (end - p < 5) error("bad unicode escape");
            unsigned cp = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
            p += 4;
            break;
          }
          default: out += *p;
        }
        ++p;
      } else {
        out += *p++;
      }
    }
    if (p >= end) error("unterminated string");
    ++p;
    return out;
  }
};

// jsonHelper.hpp:56-220 semantics
const JVal& require(const JVal& obj, const char* key) {
  const JVal* v = obj.kind == JVal::Object ? obj.find(key) : nullptr;
  if (!v) throw std::invalid_argument(std::string("JSON reader - Error : cannot found key ") + key);
  return *v;
}
[[noreturn]] void type_error(const char* key) {
  throw std::invalid_argument(std::string("JSON reader - Error : type error with key ") + key);
}
double req_double(const JVal& o, const char* key) {
  const JVal& v = require(o, key);
  if (!v.is_double()) type_error(key);
  return v.d;
}
unsigned req_uint(const JVal& o, const char* key) {
  const JVal& v = require(o, key);
  if (!v.is_uint()) type_error(key);
  return (unsigned)v.i;
}
bool req_bool(const JVal& o, const char* key) {
  const JVal& v = require(o, key);
  if (v.kind != JVal::Bool) type_error(key);
  return v.b;
}
const std::string& req_string(const JVal& o, const char* key) {
  const JVal& v = require(o, key);
  if (v.kind != JVal::String) type_error(key);
  return v.s;
}
const JVal& req_array(const JVal& o, const char* key) {
  const JVal& v = require(o, key);
  if (v.kind != JVal::Array) type_error(key);
  return v;
}
// getVectorFromArray (scene_building.cpp:302-318)
void vec3(const JVal& a, double* out) {
  if (a.a.size() != 3u) throw std::invalid_argument("JSON reader - Error : Array representing vector must be of size 3");
  for (int k = 0; k < 3; ++k) {
    if (!a.a[k].is_double())
      throw std::invalid_argument("JSON reader - Error : Array representing vector must contain doubles");
    out[k] = a.a[k].d;
  }
}

std::string read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::ios_base::failure("Couldn't open file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

JVal load_json(const std::string& path) {
  const std::string text = read_file(path);
  JParser jp(text);
  return jp.parse();
}

std::string dir_of(const std::string& path) {
  size_t k = path.find_last_of('/');
  return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

std::string resolve(const std::string& base_dir, const std::string& p) {
  if (!p.empty() && p[0] == '/') return p;
  std::string cand = base_dir + "/" + p;
  std::ifstream f(cand);
  if (f) return cand;
  return p;
}

// ---------------------------------------------------------------- OBJ
// Vertices "v x y z" (rounded through float), faces "f a[/b[/c]] ..."
// (1-based or negative relative indices, polygons fanned into triangles).
void read_obj(const std::string& path, std::vector<double>& pos, std::vector<int>& tris) {
  std::ifstream f(path);
  if (!f) throw std::ios_base::failure("Could not load obj file: " + path);
  pos.clear();
  tris.clear();
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ls(line);
    std::string tag;
    if (!(ls >> tag)) continue;
    if (tag == "v") {
      double x[3];
      std::string t;
      for (int k = 0; k < 3; ++k) {
        if (!(ls >> t)) throw std::invalid_argument("malformed vertex line in " + path);
        char* e = nullptr;
        double d = std::strtod(t.c_str(), &e);
        if (e == t.c_str()) throw std::invalid_argument("malformed vertex line in " + path);
        x[k] = (double)(float)d;
      }
      pos.insert(pos.end(), x, x + 3);
    } else if (tag == "f") {
      std::vector<int> idx;
      std::string t;
      const int nv = (int)(pos.size() / 3);
      while (ls >> t) {
        int i = std::atoi(t.c_str());
        if (i == 0) throw std::invalid_argument("malformed face in " + path);
        i = i > 0 ? i - 1 : nv + i;
        idx.push_back(i);
      }
      if (idx.size() < 3) throw std::invalid_argument("face with fewer than 3 vertices in " + path);
      for (size_t k = 1; k + 1 < idx.size(); ++k) {
        tris.push_back(idx[0]);
        tris.push_back(idx[k]);
        tris.push_back(idx[k + 1]);
      }
    }
  }
  const int nv = (int)(pos.size() / 3);
  for (int x : tris)
    if (x < 0 || x >= nv) throw std::invalid_argument("face index out of range in " + path);
}

}  // namespace

struct pdf_log {
  std::vector<int> kinds;
  std::vector<std::vector<int32_t>> vertices;
  std::vector<pdf_log_entry> entries;
};

struct pdf_scene {
  std::vector<double> rest, pos;
  std::vector<int> tris;
  std::vector<pdf_mesh_desc> meshes;
  std::vector<pdf_obstacle> obstacles;
  std::vector<std::vector<double>> ob_v;
  std::vector<std::vector<int>> ob_t;
  std::vector<int> pin_v;
  std::vector<double> pin_p, pin_w;
  std::vector<double> friction;
  int n_materials = 0;
};

extern "C" {

int pdf_scene_load_json(const char* json_path, pdf_scene** out) {
  if (!out || !json_path) return PDF_INVALID_ARG;
  *out = nullptr;
  std::unique_ptr<pdf_scene> sc(new pdf_scene());
  try {
    const JVal root = load_json(json_path);
    if (root.kind != JVal::Object) throw std::invalid_argument("JSON reader - Error : root must be an object");
    const std::string base = dir_of(json_path);
    // friction table (scene_building.cpp:77-103)
    const JVal& fr = req_array(root, "Friction coefficients");
    const size_t nm = fr.a.size();
    sc->n_materials = (int)nm;
    sc->friction.assign(nm * nm, 0.);
    for (size_t i = 0; i < nm; ++i) {
      if (fr.a[i].kind != JVal::Array || fr.a[i].a.size() != nm)
        throw std::invalid_argument("JSON reader - Error : Friction coefficients must be a square matrix");
      for (size_t j = 0; j < nm; ++j) {
        if (!fr.a[i].a[j].is_double())
          throw std::invalid_argument("JSON reader - Error : Friction coefficients must be a square matrix of double");
        sc->friction[i * nm + j] = fr.a[i].a[j].d;
      }
    }
    // meshes (scene_building.cpp:105-162)
    const JVal& ms = req_array(root, "Meshes");
    for (const JVal& mo : ms.a) {
      std::string file = resolve(base, req_string(mo, "Obj filename"));
      std::vector<double> p;
      std::vector<int> t;
      read_obj(file, p, t);
      pdf_mesh_desc md{};
      md.vertex_offset = (int)(sc->rest.size() / 3);
      md.n_vertices = (int)(p.size() / 3);
      md.triangle_offset = (int)(sc->tris.size() / 3);
      md.n_triangles = (int)(t.size() / 3);
      md.area_density = req_double(mo, "Area Density");
      md.bending = req_double(mo, "Bending");
      md.stretching = req_double(mo, "Stretching");
      md.material = (int)req_uint(mo, "Material Identifier");
      sc->rest.insert(sc->rest.end(), p.begin(), p.end());
      for (int x : t) sc->tris.push_back(x + md.vertex_offset);
      if (mo.find("Current state obj filename")) {
        std::string cf = resolve(base, req_string(mo, "Current state obj filename"));
        std::vector<double> cp;
        std::vector<int> ct;
        read_obj(cf, cp, ct);
        if (cp.size() != p.size()) throw std::invalid_argument("current state has a different vertex count");
        sc->pos.insert(sc->pos.end(), cp.begin(), cp.end());
      } else {
        sc->pos.insert(sc->pos.end(), p.begin(), p.end());
      }
      // extension: attachment constraints {"Vertex": i, "Weight": w}
      if (const JVal* at = mo.find("Attachments")) {
        if (at->kind != JVal::Array) type_error("Attachments");
        for (const JVal& a : at->a) {
          unsigned v = req_uint(a, "Vertex");
          double w = req_double(a, "Weight");
          if ((int)v >= md.n_vertices) throw std::invalid_argument("attachment vertex out of range");
          int g = md.vertex_offset + (int)v;
          sc->pin_v.push_back(g);
          sc->pin_w.push_back(w);
          for (int k = 0; k < 3; ++k) sc->pin_p.push_back(sc->pos[3 * (size_t)g + k]);
        }
      }
      sc->meshes.push_back(md);
    }
    // obstacles (scene_building.cpp:164-202, 279-295)
    const JVal& obs = req_array(root, "Obstacles");
    for (const JVal& oo : obs.a) {
      const std::string& type = req_string(oo, "Type");
      pdf_obstacle ob{};
      ob.mesh = -1;  // the reference's obstacles act on every dynamic mesh
      std::vector<double> ov;
      std::vector<int> ot;
      if (type == "Sphere") {
        ob.type = PDF_OBSTACLE_SPHERE;
        vec3(req_array(oo, "Position"), ob.center);
        ob.radius = req_double(oo, "Radius");
        ob.material = (int)req_uint(oo, "Material Identifier");
      } else if (type == "Plane") {
        ob.type = PDF_OBSTACLE_PLANE;
        vec3(req_array(oo, "Point"), ob.point);
        vec3(req_array(oo, "Normal"), ob.normal);
        ob.material = (int)req_uint(oo, "Material Identifier");
      } else if (type == "Mesh") {
        ob.type = PDF_OBSTACLE_MESH;
        read_obj(resolve(base, req_string(oo, "Path")), ov, ot);
        ob.threshold = req_double(oo, "Threshold");
        ob.material = (int)req_uint(oo, "Material Identifier");
      } else if (type == "Rotating Sphere") {
        ob.type = PDF_OBSTACLE_ROTATING_SPHERE;
        ob.radius = req_double(oo, "Radius");
        vec3(req_array(oo, "Position"), ob.center);
        vec3(req_array(oo, "Rotation Axe"), ob.axis);
        ob.angular_speed = req_double(oo, "Radial Speed");
        ob.rotation_start_time = req_double(oo, "Rotation Start Time");
        ob.material = (int)req_uint(oo, "Material Identifier");
      } else if (type == "Axis Aligned Box") {
        // getStaticAxisAlignedBoxFromObject (src/scene_building.cpp:205-211)
        ob.type = PDF_OBSTACLE_BOX;
        vec3(req_array(oo, "Position"), ob.center);
        ob.material = (int)req_uint(oo, "Material Identifier");
        vec3(req_array(oo, "Size"), ob.size);
      } else if (type == "Moving Mesh") {
        // getMovingMeshFromObject (src/scene_building.cpp:248-276): key frame f
        // is "<Obj Prefix><f, zero-padded to Suffix Size>.obj" at time
        // f * "Time Between Frame".  Every key frame is read here, at load
        // time (the reference reads them as its clock reaches them).
        ob.type = PDF_OBSTACLE_MOVING_MESH;
        const std::string prefix = req_string(oo, "Obj Prefix");
        const uint64_t suffix = req_uint(oo, "Suffix Size");
        const uint64_t frames = req_uint(oo, "Number Frame");
        ob.material = (int)req_uint(oo, "Material Identifier");
        ob.frame_interval = req_double(oo, "Time Between Frame");
        ob.threshold = req_double(oo, "Collision tolerance");
        if (frames < 2) throw std::invalid_argument("Moving Mesh needs at least two frames");
        if (frames > (1u << 20)) throw std::invalid_argument("Moving Mesh frame count too large");
        ob.n_frames = (int)frames;
        std::vector<double> fv;
        std::vector<int> ft;
        for (uint64_t f = 0; f < frames; ++f) {
          std::ostringstream name;
          name << prefix;
          if (suffix > 0) name << std::setfill('0') << std::setw((int)suffix);
          name << f << ".obj";
          read_obj(resolve(base, name.str()), fv, ft);
          if (f == 0) {
            ot = ft;
          } else if (fv.size() != ov.size() / f) {
            throw std::invalid_argument("Moving Mesh key frame " + name.str() + " has a different vertex count");
          }
          ov.insert(ov.end(), fv.begin(), fv.end());
        }
      } else {
        throw std::invalid_argument("JSON reader - Error : Invalid type for static object type");
      }
      if (ob.material < 0 || ob.material >= sc->n_materials)
        throw std::invalid_argument("obstacle material out of range");
      sc->obstacles.push_back(ob);
      sc->ob_v.push_back(std::move(ov));
      sc->ob_t.push_back(std::move(ot));
    }
  } catch (const std::ios_base::failure& e) {
    g_load_error = e.what();
    return PDF_IO_ERROR;
  } catch (const std::exception& e) {
    g_load_error = e.what();
    return PDF_INVALID_ARG;
  }
  for (size_t k = 0; k < sc->obstacles.size(); ++k) {
    if (sc->obstacles[k].type == PDF_OBSTACLE_MESH || sc->obstacles[k].type == PDF_OBSTACLE_MOVING_MESH) {
      const size_t frames = sc->obstacles[k].type == PDF_OBSTACLE_MOVING_MESH ? sc->obstacles[k].n_frames : 1;
      sc->obstacles[k].n_vertices = (int)(sc->ob_v[k].size() / 3 / frames);
      sc->obstacles[k].n_triangles = (int)(sc->ob_t[k].size() / 3);
      sc->obstacles[k].vertices = sc->ob_v[k].data();
      sc->obstacles[k].triangles = sc->ob_t[k].data();
    }
  }
  *out = sc.release();
  return PDF_OK;
}

int pdf_scene_view(const pdf_scene* sc, pdf_scene_desc* d) {
  if (!sc || !d) return PDF_INVALID_ARG;
  std::memset(d, 0, sizeof(*d));
  d->n_vertices = (int)(sc->rest.size() / 3);
  d->rest_positions = sc->rest.data();
  d->positions = sc->pos.data();
  d->velocities = nullptr;
  d->n_triangles = (int)(sc->tris.size() / 3);
  d->triangles = sc->tris.data();
  d->n_meshes = (int)sc->meshes.size();
  d->meshes = sc->meshes.data();
  d->n_pins = (int)sc->pin_v.size();
  d->pin_vertices = sc->pin_v.data();
  d->pin_positions = sc->pin_p.data();
  d->pin_weights = sc->pin_w.data();
  d->n_obstacles = (int)sc->obstacles.size();
  d->obstacles = sc->obstacles.data();
  d->n_materials = sc->n_materials;
  d->friction = sc->friction.data();
  return PDF_OK;
}

void pdf_scene_free(pdf_scene* sc) { delete sc; }

int pdf_params_load_json(const char* json_path, pdf_params* out, int32_t* frame_number, int32_t* steps_per_frame) {
  if (!json_path || !out) return PDF_INVALID_ARG;
  try {
    const JVal root = load_json(json_path);
    const JVal& pv = require(root, "Parameters");
    pdf_params p;
    pdf_params_default(&p);
    unsigned frames = req_uint(pv, "Frame number");
    p.local_global_iterations = (int)req_uint(pv, "LocalGlobal");
    p.time_step = req_double(pv, "Timestep");
    unsigned spf = req_uint(pv, "Steps per frame");
    p.self_collision = req_bool(pv, "Self-collision") ? 1 : 0;
    p.self_collision_tolerance = p.self_collision ? req_double(pv, "Self-collision tolerance") : 0.;
    const JVal& g = req_array(pv, "Gravity");
    if (g.a.size() < 3) throw std::invalid_argument("Gravity must have 3 components");
    for (int k = 0; k < 3; ++k) {
      if (!g.a[k].is_number()) type_error("Gravity");
      p.gravity[k] = g.a[k].num();
    }
    // optional, any error falls back to 0 (simulation_building.cpp:68-75)
    p.air_damping = 0.;
    const JVal* ad = pv.find("Air damping");
    if (ad && ad->is_double()) p.air_damping = ad->d;
    *out = p;
    if (frame_number) *frame_number = (int32_t)frames;
    if (steps_per_frame) *steps_per_frame = (int32_t)spf;
  } catch (const std::ios_base::failure& e) {
    g_load_error = e.what();
    return PDF_IO_ERROR;
  } catch (const std::exception& e) {
    g_load_error = e.what();
    return PDF_INVALID_ARG;
  }
  return PDF_OK;
}

int pdf_log_load_json(const char* json_path, pdf_log** out) {
  if (!json_path || !out) return PDF_INVALID_ARG;
  *out = nullptr;
  try {
    const JVal root = load_json(json_path);
    if (root.kind != JVal::Object) throw std::invalid_argument("JSON reader - Error : root must be an object");
    std::unique_ptr<pdf_log> lg(new pdf_log);
    const JVal* la = root.find("log");
    if (la) {
      const JVal& arr = req_array(root, "log");
      for (const JVal& lo : arr.a) {
        // getLogTypeFromObject (log_building.cpp:73-87), STRING_TO_LOG_TYPE
        const std::string& kind = req_string(lo, "type");
        int k;
        if (kind == "position")
          k = PDF_LOG_POSITION;
        else if (kind == "velocity")
          k = PDF_LOG_VELOCITY;
        else
          throw std::invalid_argument("Log type \"" + kind + "\" is unsupported");
        // getIndicesFromArray (log_building.cpp:120-129)
        std::vector<int32_t> idx;
        for (const JVal& x : req_array(lo, "vertices").a) {
          if (x.kind != JVal::Int || x.i < 0 || x.i > 0x7fffffffLL) type_error("vertices");
          idx.push_back((int32_t)x.i);
        }
        lg->kinds.push_back(k);
        lg->vertices.push_back(std::move(idx));
      }
    }
    lg->entries.resize(lg->kinds.size());
    for (size_t e = 0; e < lg->kinds.size(); ++e) {
      lg->entries[e].kind = lg->kinds[e];
      lg->entries[e].n_vertices = (int32_t)lg->vertices[e].size();
      lg->entries[e].vertices = lg->vertices[e].data();
    }
    *out = lg.release();
  } catch (const std::ios_base::failure& e) {
    g_load_error = e.what();
    return PDF_IO_ERROR;
  } catch (const std::exception& e) {
    g_load_error = e.what();
    return PDF_INVALID_ARG;
  }
  return PDF_OK;
}

int pdf_log_view(const pdf_log* lg, int32_t* n_entries, const pdf_log_entry** entries) {
  if (!lg) return PDF_INVALID_ARG;
  if (n_entries) *n_entries = (int32_t)lg->entries.size();
  if (entries) *entries = lg->entries.data();
  return PDF_OK;
}

void pdf_log_free(pdf_log* lg) { delete lg; }

}  // extern "C"
