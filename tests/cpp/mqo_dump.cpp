// Dumps what include/xyzgpu_mqo.hpp makes of a scene file, in the form the
// reference's Triangle stores it, for comparison with the reference's own
// loader (tests/test_mqo.py).  No GPU is needed (the spectral tables of
// libxyzgpu.so are host code).
//
//   mqo_dump <scene.mqo | mesh.ply> <out_prefix>
//       out_prefix.geo    21 float32 per triangle: v0, e1, e2, ng, n0, s1, s2
//       out_prefix.mat    int32 material per triangle
//       out_prefix.key    int32 Morton key per triangle
//       out_prefix.mats   5 float32 per material: kind (the reference's
//                         Bsdf::What: 0 Lambert, 1 mirror, 3 metal, 4 light),
//                         albedo XYZ, shininess
//       out_prefix.cam    6 float32: eye, at
//   mqo_dump --ply2mqo <mesh.ply> <out.mqo>    PlyToMqo's document
//   mqo_dump --desc <scene.mqo | mesh.ply> <out_prefix>
//       the arrays of the C ABI's scene description: .pos (3 float32 per
//       vertex), .nrm (3 float32 per vertex, or empty), .tri (3 int32 per
//       triangle), .mat, .alb (3 float32 per material), .light, .kind
//       (XYZGPU_MATERIAL_*), .shin, .power (the reference's light power XYZ)
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "xyzgpu_mqo.hpp"

template <class T>
static void put(const std::string &path, const std::vector<T> &v) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char *>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

int main(int argc, char **argv) {
  if (argc == 4 && std::string(argv[1]) == "--ply2mqo") {
    std::ifstream in(argv[2], std::ios::binary);
    std::string text, err;
    if (!xyzgpu::PlyToMqo(in, &text, &err)) {
      std::fprintf(stderr, "%s\n", err.c_str());
      return 1;
    }
    std::ofstream(argv[3], std::ios::binary) << text;
    return 0;
  }
  bool const desc = argc == 4 && std::string(argv[1]) == "--desc";
  if (argc != 3 && !desc) return 2;
  std::string const path = argv[desc ? 2 : 1], pre = argv[desc ? 3 : 2];
  std::ifstream in(path, std::ios::binary);
  xyzgpu::MqoScene sc;
  std::string err;
  bool const ply = path.size() > 4 && path.compare(path.size() - 4, 4, ".ply") == 0;
  if (!(ply ? xyzgpu::LoadPly(in, &sc, &err) : xyzgpu::LoadMqo(in, &sc, &err))) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  if (desc) {
    float power[3];
    xyzgpu::ReferenceLightPowerXYZ(power);
    xyzgpu_scene_desc const d = sc.Desc(power);
    int const nm = d.n_materials;
    put(pre + ".pos", sc.positions);
    put(pre + ".nrm", sc.normals);
    put(pre + ".tri", sc.triangles);
    put(pre + ".mat", sc.tri_material);
    put(pre + ".alb", std::vector<float>(d.albedo_xyz, d.albedo_xyz + 3 * nm));
    put(pre + ".light", std::vector<int32_t>(d.is_light, d.is_light + nm));
    put(pre + ".kind", std::vector<int32_t>(d.material_kind, d.material_kind + nm));
    put(pre + ".shin", std::vector<float>(d.shininess, d.shininess + nm));
    put(pre + ".power", std::vector<float>(power, power + 3));
    return 0;
  }
  std::vector<float> geo;
  auto P = [&](int v, int c) { return sc.positions[3 * v + c]; };
  auto N = [&](int v, int c) { return sc.normals[3 * v + c]; };
  for (size_t t = 0; t < sc.tri_material.size(); ++t) {
    int const a = sc.triangles[3 * t], b = sc.triangles[3 * t + 1], c = sc.triangles[3 * t + 2];
    float v0[3], e1[3], e2[3], ng[3], n0[3], s1[3], s2[3];
    for (int k = 0; k < 3; ++k) {
      v0[k] = P(a, k);
      e1[k] = P(b, k) - P(a, k);
      e2[k] = P(c, k) - P(a, k);
    }
    ng[0] = e2[1] * e1[2] - e2[2] * e1[1];
    ng[1] = e2[2] * e1[0] - e2[0] * e1[2];
    ng[2] = e2[0] * e1[1] - e2[1] * e1[0];
    float const s = 1.0f / std::sqrt(ng[0] * ng[0] + ng[1] * ng[1] + ng[2] * ng[2]);
    for (float &x : ng) x *= s;
    for (int k = 0; k < 3; ++k) {
      if (sc.normals.empty()) {
        n0[k] = ng[k];
        s1[k] = s2[k] = 0.0f;
      } else {
        n0[k] = N(a, k);
        s1[k] = N(b, k) - N(a, k);
        s2[k] = N(c, k) - N(a, k);
      }
    }
    for (const float *v : {v0, e1, e2, ng, n0, s1, s2}) geo.insert(geo.end(), v, v + 3);
  }
  std::vector<float> mats;
  for (auto const &m : sc.materials) {
    float const kind = m.light ? 4.0f : (m.kind == XYZGPU_MATERIAL_MIRROR ? 1.0f : (m.kind == XYZGPU_MATERIAL_METAL ? 3.0f : 0.0f));
    mats.insert(mats.end(), {kind, m.albedo[0], m.albedo[1], m.albedo[2], m.kind == XYZGPU_MATERIAL_METAL ? m.shininess : 0.0f});
  }
  put(pre + ".geo", geo);
  put(pre + ".mat", sc.tri_material);
  put(pre + ".key", sc.morton);
  put(pre + ".mats", mats);
  put(pre + ".cam", std::vector<float>{sc.eye[0], sc.eye[1], sc.eye[2], sc.at[0], sc.at[1], sc.at[2]});
  return 0;
}
