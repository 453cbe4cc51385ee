// Command-line harness around the reference's MQO loader (Scene::Load,
// xyz/core/scene_mqo.cpp, inside oracle/_ref/libxyzref_pinhole.so): loads a
// document and dumps the scene it builds.  TEST INFRASTRUCTURE: only tests/
// run it, in a process of its own (the loader's iostreams must not share a
// process with another C++ runtime).
//   xyzref_mqo <scene.mqo> <out_prefix>
//     .geo  21 float32 per triangle in its order (v0, e1, e2, ng, n0, s1, s2)
//     .mat  int32 material per triangle
//     .mats int32 kind (Bsdf::What), then 3 float32 albedo, 1 float32 shininess per material
//     .cam  6 float32: eye, at
#include <cstdio>
#include <string>
#include <vector>

extern "C" {
int xyzref_load_mqo(const char *path);
void xyzref_mqo_counts(int *n_tris, int *n_mats, int *n_lights);
void xyzref_mqo_triangles(float *geo, int *mat);
void xyzref_mqo_materials(int *kind, float *albedo, float *shininess);
void xyzref_mqo_camera(float eye[3], float at[3]);
}

template <class T>
static bool put(const std::string &path, const std::vector<T> &v) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool const ok = std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
  return std::fclose(f) == 0 && ok;
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  if (xyzref_load_mqo(argv[1]) < 0) return 3;
  int nt = 0, nm = 0, nl = 0;
  xyzref_mqo_counts(&nt, &nm, &nl);
  std::vector<float> geo(21 * static_cast<size_t>(nt)), alb(3 * static_cast<size_t>(nm)), shin(nm), cam(6);
  std::vector<int> mat(nt), kind(nm);
  xyzref_mqo_triangles(geo.data(), mat.data());
  xyzref_mqo_materials(kind.data(), alb.data(), shin.data());
  xyzref_mqo_camera(cam.data(), cam.data() + 3);
  std::string const pre = argv[2];
  return put(pre + ".geo", geo) && put(pre + ".mat", mat) && put(pre + ".kind", kind) && put(pre + ".alb", alb) &&
                 put(pre + ".shin", shin) && put(pre + ".cam", cam)
             ? 0
             : 4;
}
