// Scene files of the reference renderer for the xyzgpu C ABI (host C++,
// header-only): Metasequoia documents (.mqo), which the reference loads with
// Scene::Load (xyz/core/scene_mqo.cpp:547-696), and PLY meshes, which it
// converts to .mqo with its ply2mqo tool (ply2mqo/main.cpp).
//
//   xyzgpu::MqoScene sc;
//   std::string err;
//   if (!xyzgpu::LoadMqo(std::ifstream("room.mqo"), &sc, &err)) ...
//   xyzgpu_scene_desc d = sc.Desc(power_xyz);  // then xyzgpu_scene_create
//
// What the reference's loader does, and this one with it:
//  * Scene chunk: camera from `pos`, `lookat`, `head`, `pich` (pitch about x,
//    then heading - pi about y, centimetres to metres); the camera looks from
//    lookat + pos at lookat.
//  * Material chunk: emi(1) is a light; an opaque colour (col alpha 1) with
//    spc(1) and power(100) a mirror, with spc(1) and another power > 0 a metal
//    of that exponent, otherwise Lambert.  Albedo: a material whose name holds
//    "mcc-<patch>" takes the ColorChecker patch's XYZ (first match in the
//    reference's order, so "mcc-orange-yellow" is "mcc-orange"), otherwise
//    (col * spc)^2.2 converted by CCIR 601-1; clamped to [0, 1].  A document
//    whose Material chunk is empty gets one white Lambert material.  A
//    transparent material (glass in the reference) is refused: the path
//    tracer has no glass.
//  * Object chunks: invisible objects are skipped; vertices in centimetres
//    become metres; faces of three vertices with their material; a face of
//    another size leaves the default triangle (vertices 0, 0, 0, material 0)
//    as the reference's does.  Objects with shading 1 get vertex normals
//    averaged over their faces with weights 1 - angle / pi; flat objects use
//    the face normal.
//  * The triangles are then sorted by a Morton code of their bounding-box
//    centres over the scene box (scene_mqo.cpp:676-692), stably here (the
//    reference's std::sort leaves equal codes in any order).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <istream>
#include <sstream>
#include <string>
#include <vector>

#include "xyzgpu.h"

namespace xyzgpu {

struct MqoMaterial {
  std::string name;
  int kind = XYZGPU_MATERIAL_LAMBERT;  // XYZGPU_MATERIAL_* for non-lights
  bool light = false;
  float albedo[3] = {0, 0, 0};         // XYZ
  float shininess = 1.0f;              // metal exponent
};

struct MqoScene {
  std::vector<float> positions;        // 3 per vertex (metres)
  std::vector<float> normals;          // 3 per vertex, or empty (all objects flat)
  std::vector<int32_t> triangles;      // 3 vertex indices per triangle, in Morton order
  std::vector<int32_t> tri_material;
  std::vector<MqoMaterial> materials;
  std::vector<int32_t> morton;         // Morton key of each triangle (non-decreasing)
  bool has_camera = false;
  float eye[3] = {0.0f, 1.0f, 4.0f};   // ThinLensCamera defaults (thinlenscamera.cpp:20-28)
  float at[3] = {0.0f, 1.0f, 0.0f};

  // Arrays of the C ABI's scene description (pointers into this object).
  xyzgpu_scene_desc Desc(const float light_power_xyz[3]) {
    xyzgpu_scene_desc d;
    std::memset(&d, 0, sizeof(d));
    kind_.assign(materials.size(), 0);
    light_.assign(materials.size(), 0);
    albedo_.assign(3 * materials.size(), 0.0f);
    shin_.assign(materials.size(), 1.0f);
    for (size_t m = 0; m < materials.size(); ++m) {
      kind_[m] = materials[m].kind;
      light_[m] = materials[m].light ? 1 : 0;
      for (int c = 0; c < 3; ++c) albedo_[3 * m + c] = materials[m].albedo[c];
      shin_[m] = materials[m].shininess;
    }
    d.positions = positions.data();
    d.normals = normals.empty() ? nullptr : normals.data();
    d.n_vertices = static_cast<int>(positions.size() / 3);
    d.triangles = triangles.data();
    d.tri_material = tri_material.data();
    d.n_triangles = static_cast<int>(tri_material.size());
    d.albedo_xyz = albedo_.data();
    d.is_light = light_.data();
    d.n_materials = static_cast<int>(materials.size());
    for (int c = 0; c < 3; ++c) d.light_power_xyz[c] = light_power_xyz[c];
    d.material_kind = kind_.data();
    d.shininess = shin_.data();
    return d;
  }

 private:
  std::vector<int32_t> kind_, light_;
  std::vector<float> albedo_, shin_;
};

// The reference's light power: the Mercury-arc lamp spectrum's XYZ
// (GetLightPowerXYZ, xyz/core/config.hpp:81-95).
inline void ReferenceLightPowerXYZ(float out[3]) {
  float spd[31];
  xyzgpu_named_spectrum("light_mercury_arc_lamp", spd);
  xyzgpu_spectrum_to_xyz(spd, out);
}

namespace mqo_detail {

inline void trim(std::string &s) {
  size_t const b = s.find_first_not_of(" \t\r\n");
  if (b == std::string::npos) {
    s.clear();
    return;
  }
  s = s.substr(b, s.find_last_not_of(" \t\r\n") - b + 1);
}

// Reads lines until the braces opened on them are closed (a line that opens
// none ends the skip at once).
inline void skip_block(std::istream &in) {
  int depth = 0;
  std::string line;
  do {
    if (!std::getline(in, line)) return;
    trim(line);
    if (line.empty()) continue;
    if (line.back() == '{')
      ++depth;
    else if (line.back() == '}')
      --depth;
  } while (depth > 0);
}

inline float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

// Albedo of a material (the two branches of scene_mqo.cpp:135-298).
inline void material_xyz(const std::string &name, const float col[4], float spc, float xyz[3]) {
  // patch names in the order the reference tests them
  static const char *const kPatches[][2] = {
      {"mcc-dark-skin", "mcc_dark_skin"},         {"mcc-light-skin", "mcc_light_skin"},
      {"mcc-blue-sky", "mcc_blue_sky"},           {"mcc-foliage", "mcc_foliage"},
      {"mcc-blue-flower", "mcc_blue_flower"},     {"mcc-bluish-green", "mcc_bluish_green"},
      {"mcc-orange", "mcc_orange"},               {"mcc-purplish-blue", "mcc_purplish_blue"},
      {"mcc-moderate-red", "mcc_moderate_red"},   {"mcc-purple", "mcc_purple"},
      {"mcc-yellow-green", "mcc_yellow_green"},   {"mcc-orange-yellow", "mcc_orange_yellow"},
      {"mcc-blue", "mcc_blue"},                   {"mcc-green", "mcc_green"},
      {"mcc-red", "mcc_red"},                     {"mcc-yellow", "mcc_yellow"},
      {"mcc-magenta", "mcc_magenta"},             {"mcc-cyan", "mcc_cyan"},
      {"mcc-white", "mcc_white"},                 {"mcc-neutral-80", "mcc_neutral80"},
      {"mcc-neutral-65", "mcc_neutral65"},        {"mcc-neutral-50", "mcc_neutral50"},
      {"mcc-neutral-35", "mcc_neutral35"},        {"mcc-black", "mcc_black"}};
  bool named = false;
  for (auto const &p : kPatches)
    if (name.find(p[0]) != std::string::npos) {
      float spd[31];
      xyzgpu_named_spectrum(p[1], spd);
      xyzgpu_spectrum_to_xyz(spd, xyz);
      named = true;
      break;
    }
  if (!named) {
    // gamma 2.2 on col * spc, then CCIR601_1_RGB2XYZ (libhi/hi/image/color_space.hpp:58-67)
    float const r = std::pow(col[0] * spc, 2.2f), g = std::pow(col[1] * spc, 2.2f),
                b = std::pow(col[2] * spc, 2.2f);
    xyz[0] = 0.6069f * r + 0.1735f * g + 0.2003f * b;
    xyz[1] = 0.2989f * r + 0.5866f * g + 0.1145f * b;
    xyz[2] = 0.0000f * r + 0.0661f * g + 1.1162f * b;
  }
  for (int c = 0; c < 3; ++c) xyz[c] = clamp01(xyz[c]);
}

// One material line: "name" shader(3) col(r g b a) dif(.) amb(.) emi(.)
// spc(.) power(.) [tex(".") ...].
inline bool parse_material(std::istream &in, const std::string &line, MqoMaterial *out, std::string *err) {
  size_t const q0 = line.find('"'), q1 = q0 == std::string::npos ? q0 : line.find('"', q0 + 1);
  if (q1 == std::string::npos) {
    *err = "material line without a quoted name: " + line;
    return false;
  }
  out->name = line.substr(q0 + 1, q1 - q0 - 1);
  float col[4] = {1, 1, 1, 1}, emi = 0, spc = 0, power = 5;
  std::string rest = line.substr(q1 + 1);
  size_t pos = 0;
  while (pos < rest.size()) {
    size_t const open = rest.find('(', pos);
    if (open == std::string::npos) break;
    std::string tag = rest.substr(pos, open - pos);
    trim(tag);
    if (tag.empty()) break;
    if (tag == "tex" || tag == "aplane" || tag == "bump") {
      // the reference reads a quoted file name here and then (from the file
      // stream, not the line) up to the next ')'; textures are not used
      size_t const a = rest.find('"', open), b = a == std::string::npos ? a : rest.find('"', a + 1);
      std::string skip;
      std::getline(in, skip, ')');
      pos = b == std::string::npos ? rest.size() : b + 1;
      size_t const close = rest.find(')', pos);
      pos = close == std::string::npos ? rest.size() : close + 1;
      continue;
    }
    size_t const close = rest.find(')', open);
    if (close == std::string::npos) break;
    std::istringstream din(rest.substr(open + 1, close - open - 1));
    if (tag == "col")
      din >> col[0] >> col[1] >> col[2] >> col[3];
    else if (tag == "emi")
      din >> emi;
    else if (tag == "spc")
      din >> spc;
    else if (tag == "power")
      din >> power;
    pos = close + 1;
  }
  if (emi == 1.0f) {
    out->light = true;
  } else if (col[3] == 1.0f) {
    if (spc == 1.0f && power > 0.0f) {
      if (power == 100.0f) {
        out->kind = XYZGPU_MATERIAL_MIRROR;
      } else {
        out->kind = XYZGPU_MATERIAL_METAL;
        out->shininess = power;
        material_xyz(out->name, col, spc, out->albedo);
      }
    } else {
      material_xyz(out->name, col, spc, out->albedo);
    }
  } else {
    *err = "material \"" + out->name + "\" is transparent (glass): not part of the path tracer";
    return false;
  }
  return true;
}

struct Face {
  int v[3] = {0, 0, 0};
  int m = 0;
};

inline float length3(const float a[3]) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
inline void normalize3(float a[3]) {
  float const s = 1.0f / std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] *= s, a[1] *= s, a[2] *= s;
}

// One Object chunk (after its "Object "name" {" line).
inline bool parse_object(std::istream &in, MqoScene *sc, std::vector<std::vector<float>> *obj_normals,
                         std::vector<Face> *faces_out, size_t *vbase_out, bool *smooth_out, bool *visible_out,
                         std::string *err) {
  int visible = 0, shading = 1;
  std::vector<float> verts;
  std::vector<Face> faces;
  std::string tok, line;
  for (;;) {
    if (!(in >> tok)) {
      *err = "unterminated Object chunk";
      return false;
    }
    if (tok == "visible") {
      in >> visible;
    } else if (tok == "shading") {
      in >> shading;
    } else if (tok == "vertex") {
      if (!visible) {
        skip_block(in);
        continue;
      }
      int n = 0;
      in >> n;
      std::getline(in, line);  // " {"
      for (int i = 0; i < n; ++i) {
        std::getline(in, line);
        std::istringstream sin(line);
        float p[3] = {0, 0, 0};
        sin >> p[0] >> p[1] >> p[2];
        for (float v : p) verts.push_back(v * 0.01f);  // centimetres -> metres
      }
      std::getline(in, line);  // "}"
    } else if (tok == "face") {
      if (!visible) {
        skip_block(in);
        continue;
      }
      int n = 0;
      in >> n;
      faces.assign(static_cast<size_t>(std::max(n, 0)), Face());
      std::getline(in, line);
      for (int i = 0; i < n; ++i) {
        std::getline(in, line);
        std::replace(line.begin(), line.end(), '(', ' ');
        std::replace(line.begin(), line.end(), ')', ' ');
        std::istringstream sin(line);
        int k = 0;
        sin >> k;
        if (k != 3) continue;
        std::string tag;
        for (int j = 0; j < 3; ++j) {
          if (!(sin >> tag)) break;
          if (tag == "V") {
            sin >> faces[i].v[0] >> faces[i].v[1] >> faces[i].v[2];
          } else if (tag == "M") {
            sin >> faces[i].m;
          } else if (tag == "UV") {
            float uv;
            for (int q = 0; q < 6; ++q) sin >> uv;
          }
        }
      }
      std::getline(in, line);
    } else if (tok == "}") {
      break;
    } else {
      skip_block(in);
    }
  }
  *visible_out = visible != 0;
  if (!visible) return true;
  int const nverts = static_cast<int>(verts.size() / 3);
  for (Face const &f : faces)
    for (int v : f.v)
      if (v < 0 || v >= nverts) {
        *err = "a face refers to a vertex out of range";
        return false;
      }
  *vbase_out = sc->positions.size() / 3;
  sc->positions.insert(sc->positions.end(), verts.begin(), verts.end());
  *smooth_out = shading != 0;
  std::vector<float> normals;
  if (shading) {
    // vertex normals: face normals weighted by 1 - (corner angle) / pi
    normals.assign(verts.size(), 0.0f);
    auto P = [&](int v, int c) { return verts[3 * v + c]; };
    for (Face const &f : faces) {
      float ea[3], eb[3], ec[3];
      for (int c = 0; c < 3; ++c) {
        ea[c] = P(f.v[1], c) - P(f.v[2], c);
        eb[c] = P(f.v[2], c) - P(f.v[0], c);
        ec[c] = P(f.v[0], c) - P(f.v[1], c);
      }
      float const a = length3(ea), b = length3(eb), c = length3(ec);
      auto dot = [](const float *x, const float *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
      float const wa = static_cast<float>(std::max(0.0, 1 - 0.318309886183790671538 * std::acos(dot(eb, ec) / (b * c))));
      float const wb = static_cast<float>(std::max(0.0, 1 - 0.318309886183790671538 * std::acos(dot(ec, ea) / (c * a))));
      float const wc = static_cast<float>(std::max(0.0, 1 - 0.318309886183790671538 * std::acos(dot(ea, eb) / (a * b))));
      // NormalVector(ec, -eb) = cross(-eb, ec)
      float n[3] = {-eb[1] * ec[2] - -eb[2] * ec[1], -eb[2] * ec[0] - -eb[0] * ec[2], -eb[0] * ec[1] - -eb[1] * ec[0]};
      normalize3(n);
      float const w[3] = {wa, wb, wc};
      for (int k = 0; k < 3; ++k)
        for (int q = 0; q < 3; ++q) normals[3 * f.v[k] + q] += n[q] * w[k];
    }
    for (size_t v = 0; v < normals.size() / 3; ++v) normalize3(&normals[3 * v]);
  }
  obj_normals->push_back(normals);
  *faces_out = faces;
  return true;
}

// hi::morton_code of 12-bit cell coordinates (libhi/hi/math/math.hpp:303-317):
// bit i of x, y, z lands at bit 3i, 3i + 1, 3i + 2 of a 32-bit word.
inline int32_t morton3(int x, int y, int z) {
  uint32_t code = 0;
  for (int i = 0; i < 12; ++i) {
    uint32_t const bx = (static_cast<uint32_t>(x) >> i) & 1u, by = (static_cast<uint32_t>(y) >> i) & 1u,
                   bz = (static_cast<uint32_t>(z) >> i) & 1u;
    if (3 * i < 32) code |= bx << (3 * i);
    if (3 * i + 1 < 32) code |= by << (3 * i + 1);
    if (3 * i + 2 < 32) code |= bz << (3 * i + 2);
  }
  return static_cast<int32_t>(code);
}

}  // namespace mqo_detail

// Parses a Metasequoia text document into `sc`.  Returns false (with a
// message) on a document the reference would not load or a material this
// tracer does not have.
inline bool LoadMqo(std::istream &in, MqoScene *sc, std::string *err) {
  using namespace mqo_detail;
  *sc = MqoScene();
  std::string line, tag;
  if (!std::getline(in, line) || (trim(line), line) != "Metasequoia Document") {
    *err = "not a Metasequoia document";
    return false;
  }
  if (!std::getline(in, line) || (trim(line), line) != "Format Text Ver 1.0") {
    *err = "unsupported Metasequoia format: " + line;
    return false;
  }
  // per object: its triangles (global vertex ids), material, normals
  struct Tri {
    int v[3];
    int m;
    float n[9];
    bool smooth;
  };
  std::vector<Tri> tris;
  bool any_smooth = false, any_flat = false;
  while (in >> tag) {
    if (tag == "Scene") {
      float pos[3] = {0, 0, 400}, look[3] = {0, 100, 0}, head = 0, pitch = 0;
      int depth = 0;
      do {
        if (!std::getline(in, line)) break;
        trim(line);
        if (line.empty()) continue;
        if (line.back() == '{') {
          ++depth;
        } else if (line.back() == '}') {
          --depth;
        } else {
          std::istringstream din(line);
          std::string t;
          din >> t;
          if (t == "pos")
            din >> pos[0] >> pos[1] >> pos[2];
          else if (t == "lookat")
            din >> look[0] >> look[1] >> look[2];
          else if (t == "head")
            din >> head;
          else if (t == "pich")
            din >> pitch;
        }
      } while (depth > 0);
      // pitch (y-z), then heading - pi (z-x) (scene_mqo.cpp:598-617)
      {
        float const s = std::sin(pitch), c = std::cos(pitch);
        float const v1 = pos[1], v2 = pos[2];
        pos[1] = c * v1 + s * v2;
        pos[2] = s * v1 - c * v2;
      }
      {
        head = static_cast<float>(head - 3.14159265358979323846);
        float const s = std::sin(head), c = std::cos(head);
        float const v0 = pos[0], v2 = pos[2];
        pos[2] = c * v2 + s * v0;
        pos[0] = s * v2 - c * v0;
      }
      // (hi::basic_vector3 *= double multiplies by the float-rounded factor)
      for (int k = 0; k < 3; ++k) {
        pos[k] = pos[k] * 0.01f;
        look[k] = look[k] * 0.01f;
        sc->eye[k] = look[k] + pos[k];
        sc->at[k] = look[k];
      }
      sc->has_camera = true;
    }
    if (tag == "Material") {
      int n = 0;
      in >> n;
      if (n > 0) {
        std::getline(in, line);  // " {"
        for (int i = 0; i < n; ++i) {
          std::getline(in, line);
          MqoMaterial m;
          if (!parse_material(in, line, &m, err)) return false;
          sc->materials.push_back(m);
        }
        std::getline(in, line);  // "}"
      } else {
        MqoMaterial m;
        m.name = "(default)";
        float const col[4] = {1, 1, 1, 1};
        std::string white = "mcc-white";
        material_xyz(white, col, 0.0f, m.albedo);
        sc->materials.push_back(m);
        skip_block(in);
      }
    } else if (tag == "Object") {
      std::getline(in, line);  // "name" {
      std::vector<std::vector<float>> nrm;
      std::vector<Face> faces;
      size_t vbase = 0;
      bool smooth = false, visible = false;
      if (!parse_object(in, sc, &nrm, &faces, &vbase, &smooth, &visible, err)) return false;
      std::getline(in, line);
      if (!visible) continue;
      (smooth ? any_smooth : any_flat) = true;
      for (Face const &f : faces) {
        Tri t;
        for (int k = 0; k < 3; ++k) t.v[k] = static_cast<int>(vbase) + f.v[k];
        t.m = f.m;
        t.smooth = smooth;
        for (int k = 0; k < 3; ++k)
          for (int q = 0; q < 3; ++q) t.n[3 * k + q] = smooth ? nrm[0][3 * f.v[k] + q] : 0.0f;
        tris.push_back(t);
      }
    } else if (tag == "Eof") {
      break;
    }
  }
  for (Tri const &t : tris)
    if (t.m < 0 || t.m >= static_cast<int>(sc->materials.size())) {
      *err = "a face refers to a material out of range";
      return false;
    }
  // Morton order (scene_mqo.cpp:676-692) with the triangles' stored
  // geometry: v0, v0 + e1, v0 + e2 (e = p - v0 in float)
  auto corner = [&](const Tri &t, int k, int c) {
    float const v0 = sc->positions[3 * t.v[0] + c];
    return k == 0 ? v0 : v0 + (sc->positions[3 * t.v[k] + c] - v0);
  };
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (Tri const &t : tris)
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) {
        lo[c] = std::min(lo[c], corner(t, k, c));
        hi[c] = std::max(hi[c], corner(t, k, c));
      }
  float range[3];
  for (int c = 0; c < 3; ++c) range[c] = (hi[c] - lo[c]) * 1e-5f;
  std::vector<int32_t> key(tris.size());
  for (size_t i = 0; i < tris.size(); ++i) {
    int cell[3];
    for (int c = 0; c < 3; ++c) {
      float mn = corner(tris[i], 0, c), mx = mn;
      for (int k = 1; k < 3; ++k) {
        mn = std::min(mn, corner(tris[i], k, c));
        mx = std::max(mx, corner(tris[i], k, c));
      }
      float const centre = (mn + mx) * 0.5f;
      cell[c] = static_cast<int>((centre - lo[c]) / range[c] * 1024);
    }
    key[i] = morton3(cell[0], cell[1], cell[2]);
  }
  std::vector<size_t> order(tris.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
  // vertices: as loaded when every object is smooth or every one flat; one
  // vertex per triangle corner when they are mixed (flat corners carry the
  // face normal, the shading normal the reference's flat triangles use)
  bool const expand = any_smooth && any_flat;
  std::vector<float> pos_in = sc->positions;
  if (expand) sc->positions.clear();
  if (any_smooth && !expand) sc->normals.assign(pos_in.size(), 0.0f);
  for (size_t oi = 0; oi < order.size(); ++oi) {
    Tri const &t = tris[order[oi]];
    sc->morton.push_back(key[order[oi]]);
    sc->tri_material.push_back(t.m);
    if (!expand) {
      for (int k = 0; k < 3; ++k) {
        sc->triangles.push_back(t.v[k]);
        if (any_smooth)
          for (int q = 0; q < 3; ++q) sc->normals[3 * t.v[k] + q] = t.n[3 * k + q];
      }
      continue;
    }
    float fn[3] = {0, 0, 0};
    if (!t.smooth) {
      float e1[3], e2[3];
      for (int c = 0; c < 3; ++c) {
        e1[c] = pos_in[3 * t.v[1] + c] - pos_in[3 * t.v[0] + c];
        e2[c] = pos_in[3 * t.v[2] + c] - pos_in[3 * t.v[0] + c];
      }
      fn[0] = e2[1] * e1[2] - e2[2] * e1[1];
      fn[1] = e2[2] * e1[0] - e2[0] * e1[2];
      fn[2] = e2[0] * e1[1] - e2[1] * e1[0];
      normalize3(fn);
    }
    for (int k = 0; k < 3; ++k) {
      sc->triangles.push_back(static_cast<int32_t>(sc->positions.size() / 3));
      for (int q = 0; q < 3; ++q) {
        sc->positions.push_back(pos_in[3 * t.v[k] + q]);
        sc->normals.push_back(t.smooth ? t.n[3 * k + q] : fn[q]);
      }
    }
  }
  return true;
}

namespace ply_detail {

struct Prop {
  std::string name, type, count_type;  // count_type non-empty: a list
};
struct Element {
  std::string name;
  long count = 0;
  std::vector<Prop> props;
};

inline int type_size(const std::string &t) {
  if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
  if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
  if (t == "int" || t == "uint" || t == "float" || t == "int32" || t == "uint32" || t == "float32") return 4;
  if (t == "double" || t == "float64") return 8;
  return 0;
}

// One scalar of `type` as rply reports it (a double; ASCII through strtod).
inline bool read_value(std::istream &in, int fmt, const std::string &type, double *v) {
  if (fmt == 0) {
    std::string w;
    if (!(in >> w)) return false;
    char *end = nullptr;
    *v = std::strtod(w.c_str(), &end);
    return end && *end == 0;
  }
  int const n = type_size(type);
  unsigned char b[8];
  if (n == 0 || !in.read(reinterpret_cast<char *>(b), n)) return false;
  if (fmt == 2) std::reverse(b, b + n);  // big-endian file
  if (type == "char" || type == "int8") *v = static_cast<int8_t>(b[0]);
  else if (type == "uchar" || type == "uint8") *v = b[0];
  else if (type == "short" || type == "int16") { int16_t x; std::memcpy(&x, b, 2); *v = x; }
  else if (type == "ushort" || type == "uint16") { uint16_t x; std::memcpy(&x, b, 2); *v = x; }
  else if (type == "int" || type == "int32") { int32_t x; std::memcpy(&x, b, 4); *v = x; }
  else if (type == "uint" || type == "uint32") { uint32_t x; std::memcpy(&x, b, 4); *v = x; }
  else if (type == "float" || type == "float32") { float x; std::memcpy(&x, b, 4); *v = x; }
  else { double x; std::memcpy(&x, b, 8); *v = x; }
  return true;
}

inline std::string fmt_g(const char *f, double v) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), f, v);
  return buf;
}

}  // namespace ply_detail

// A PLY mesh (ASCII or binary; vertex x y z; faces of 3 or 4 vertex indices,
// or triangle strips) as the .mqo document the reference's ply2mqo tool writes
// for it (ply2mqo/main.cpp:158-305): its Scene chunk, one visible flat object
// "obj1", the vertices and indices printed with %g, quads kept as 4-vertex
// faces and strips as a face chunk of their triangles.  It has no Material
// chunk (LoadPly adds one).
inline bool PlyToMqo(std::istream &in, std::string *mqo_text, std::string *err) {
  using namespace ply_detail;
  std::string line;
  if (!std::getline(in, line) || (mqo_detail::trim(line), line) != "ply") {
    *err = "not a PLY file";
    return false;
  }
  int fmt = -1;
  std::vector<Element> elems;
  while (std::getline(in, line)) {
    mqo_detail::trim(line);
    std::istringstream hs(line);
    std::string w;
    hs >> w;
    if (w == "format") {
      std::string f;
      hs >> f;
      fmt = f == "ascii" ? 0 : f == "binary_little_endian" ? 1 : f == "binary_big_endian" ? 2 : -1;
    } else if (w == "element") {
      Element e;
      hs >> e.name >> e.count;
      elems.push_back(e);
    } else if (w == "property") {
      if (elems.empty()) break;
      Prop p;
      std::string t;
      hs >> t;
      if (t == "list")
        hs >> p.count_type >> p.type >> p.name;
      else
        p.type = t, hs >> p.name;
      elems.back().props.push_back(p);
    } else if (w == "end_header") {
      break;
    }
  }
  if (fmt < 0) {
    *err = "PLY header without a known format";
    return false;
  }
  std::string o =
      "Metasequoia Document\nFormat Text Ver 1.0\n\nScene {\n  pos 0.0000 0.0000 400.0000\n"
      "  lookat 0.0000 000.0000 0.0000\n  head 0.0000\n  pich 0.0000\n  ortho 0\n  zoom2 6.0000\n"
      "  amb 0.250 0.250 0.250\n}\nObject \"obj1\" {\n  depth 0\n  folding 0\n"
      "  scale 1.000000 1.000000 1.000000\n  rotation 0.000000 0.000000 0.000000\n"
      "  translation 0.000000 0.000000 0.000000\n  visible 15\n  locking 0\n  shading 0\n"
      "  facet 59.5\n  color 0.898 0.498 0.698\n  color_type 0\n";
  for (Element const &e : elems) {
    bool const is_vertex = e.name == "vertex", is_face = e.name == "face", is_strip = e.name == "tristrips";
    std::vector<int> strip;
    for (long i = 0; i < e.count; ++i) {
      for (Prop const &p : e.props) {
        if (p.count_type.empty()) {
          double v;
          if (!read_value(in, fmt, p.type, &v)) {
            *err = "PLY data ends early";
            return false;
          }
          if (is_vertex && (p.name == "x" || p.name == "y" || p.name == "z")) {
            if (p.name == "x") {
              if (i == 0) o += "  vertex " + std::to_string(e.count) + " {\n";
              o += fmt_g("    %g", v);
            } else if (p.name == "y") {
              o += fmt_g(" %g ", v);
            } else {
              o += fmt_g("%g\n", v);
              if (i + 1 >= e.count) o += "  }\n";
            }
          }
          continue;
        }
        double nd;
        if (!read_value(in, fmt, p.count_type, &nd)) {
          *err = "PLY data ends early";
          return false;
        }
        long const n = static_cast<long>(nd);
        std::vector<double> vals(static_cast<size_t>(std::max(0L, n)));
        for (long k = 0; k < n; ++k)
          if (!read_value(in, fmt, p.type, &vals[k])) {
            *err = "PLY data ends early";
            return false;
          }
        if (is_face && p.name == "vertex_indices") {
          if (n != 3 && n != 4) {
            *err = "a PLY face has neither 3 nor 4 vertices";
            return false;
          }
          if (i == 0) o += "  face " + std::to_string(e.count) + " {\n";
          o += "    " + std::to_string(n) + " V(";
          for (long k = 0; k < n; ++k) o += fmt_g(k + 1 < n ? "%g " : "%g)\n", vals[k]);
          if (i + 1 >= e.count) o += "  }\n";
        } else if (is_strip && p.name == "vertex_indices") {
          strip.assign(vals.begin(), vals.end());
        }
      }
    }
    if (is_strip && !strip.empty()) {
      // the strip's triangles, every other one flipped (ply2mqo/main.cpp:100-150)
      long nfaces = 0;
      int nv = 0;
      for (int v : strip) {
        if (v < 0)
          nv = 0;
        else if (nv < 2)
          ++nv;
        else
          ++nfaces;
      }
      o += "  face " + std::to_string(nfaces) + " {\n";
      nv = 0;
      bool flip = false;
      char buf[96];
      for (size_t k = 0; k < strip.size(); ++k) {
        if (strip[k] < 0) {
          nv = 0;
          flip = false;
        } else if (nv < 2) {
          ++nv;
        } else {
          if (flip)
            std::snprintf(buf, sizeof(buf), "    3 V(%d %d %d)\n", strip[k - 2], strip[k - 1], strip[k]);
          else
            std::snprintf(buf, sizeof(buf), "    3 V(%d %d %d)\n", strip[k - 1], strip[k - 2], strip[k]);
          o += buf;
          flip = !flip;
        }
      }
      o += "  }\n";
    }
  }
  o += "}\nEof\n";
  *mqo_text = o;
  return true;
}

// A PLY mesh as a scene: the document PlyToMqo writes, with one Material
// chunk of a white Lambert material ("mcc-white") added ahead of the object.
inline bool LoadPly(std::istream &in, MqoScene *sc, std::string *err) {
  std::string text;
  if (!PlyToMqo(in, &text, err)) return false;
  size_t const at = text.find("Object \"obj1\"");
  text.insert(at, "Material 1 {\n\t\"mcc-white\" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) "
                  "emi(0.000) spc(0.000) power(5.00)\n}\n");
  std::istringstream mqo(text);
  return LoadMqo(mqo, sc, err);
}

}  // namespace xyzgpu
