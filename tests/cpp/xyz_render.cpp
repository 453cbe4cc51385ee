// Drives the GPU path tracer through the C++ host layer (include/xyzgpu_scene.hpp)
// the way the reference's shell drives xyz::Scene and PathTracer
// (xyz/core/shell.cpp:204-497: load, set eye/at/dim, ren).
//
//   xyz_render <scene_dir> <out> <spp> <interval> <seed> <max_depth>
//              [--guided | --checkpoint <file>]
//       scene_dir holds positions.f32 triangles.i32 material.i32 albedo.f32
//       is_light.i32 power.f32 camera.f32 (eye, at, film, focal, F, pinhole)
//       dims.i32 (W, H) and, optionally, normals.f32; writes the film / spp to
//       `out` (.pfm, .float, .hdr or .bmp) after every pass and prints
//       "passes N spp S sum X"; --guided renders with GuidedPathTracer (the
//       first quarter of the samples train the guide); --checkpoint saves the
//       render after every pass and resumes from the file if it exists.
//   xyz_render --film-selftest <out.pfm> <out.float>
//       writes a synthetic 3 x 2 film with both writers (no GPU needed).
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "xyzgpu_scene.hpp"

template <class T>
static std::vector<T> read_all(const std::string &path, bool required = true) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) {
    if (required) {
      std::fprintf(stderr, "cannot read %s\n", path.c_str());
      std::exit(2);
    }
    return {};
  }
  std::streamsize const n = in.tellg();
  in.seekg(0);
  std::vector<T> v(static_cast<size_t>(n) / sizeof(T));
  in.read(reinterpret_cast<char *>(v.data()), n);
  return v;
}

int main(int argc, char **argv) {
  if (argc == 4 && std::string(argv[1]) == "--film-selftest") {
    xyzgpu::ImageFilm film(3, 2);
    for (int i = 0; i < 18; ++i) film.data()[i] = 0.5f * static_cast<float>(i) - 2.0f;
    film.data()[17] = NAN;
    // an extension no writer takes is refused (.hdr and .bmp go through the
    // device encoders, which the film I/O tests cover)
    bool const ok = film.Save(argv[2], 2.0f) && film.Save(argv[3], 2.0f) && !film.Save("x.unknown", 2.0f);
    return ok ? 0 : 1;
  }
  bool const guided = argc == 8 && std::string(argv[7]) == "--guided";
  bool const ckpt = argc == 9 && std::string(argv[7]) == "--checkpoint";
  if (argc != 7 && !guided && !ckpt) {
    std::fprintf(stderr,
                 "usage: xyz_render <scene_dir> <out> <spp> <interval> <seed> <max_depth> "
                 "[--guided | --checkpoint <file>]\n");
    return 2;
  }
  std::string const dir = argv[1];
  auto pos = read_all<float>(dir + "/positions.f32");
  auto tri = read_all<int32_t>(dir + "/triangles.i32");
  auto mat = read_all<int32_t>(dir + "/material.i32");
  auto alb = read_all<float>(dir + "/albedo.f32");
  auto lit = read_all<int32_t>(dir + "/is_light.i32");
  auto pw = read_all<float>(dir + "/power.f32");
  auto cam = read_all<float>(dir + "/camera.f32");
  auto dims = read_all<int32_t>(dir + "/dims.i32");
  auto nrm = read_all<float>(dir + "/normals.f32", false);
  try {
    xyzgpu::Scene scene;
    scene.Load(pos, tri, mat, alb, lit, pw.data(), nrm);   // load
    scene.Build();
    scene.ThinLensCamera().MoveTo(cam[0], cam[1], cam[2]);  // set eye
    scene.ThinLensCamera().LookAt(cam[3], cam[4], cam[5]);  // set at
    scene.ThinLensCamera().SetFilmSize(cam[6]);
    scene.ThinLensCamera().SetFocalLength(cam[7]);
    scene.ThinLensCamera().SetFNumber(cam[8]);
    scene.ThinLensCamera().SetPinhole(cam[9] > 0.5f);
    scene.SetDimension(dims[0], dims[1]);                    // set dim
    xyzgpu::ImageFilm film;
    int passes = 0;
    std::string const out = argv[2];
    auto on_pass = [&](const xyzgpu::ImageFilm &f, int s) {
      ++passes;
      return f.Save(out, static_cast<float>(s));
    };
    int spp = 0;
    if (guided) {
      xyzgpu::GuidedPathTracer gpt;                          // ren, guided
      gpt.seed = std::strtoull(argv[5], nullptr, 10);
      gpt.max_depth = std::atoi(argv[6]);
      spp = gpt.run(scene, &film, std::atoi(argv[3]), std::atoi(argv[4]), on_pass);
    } else {
      xyzgpu::PathTracer pt;                                 // ren
      pt.seed = std::strtoull(argv[5], nullptr, 10);
      pt.max_depth = std::atoi(argv[6]);
      if (ckpt) pt.checkpoint = argv[8];
      spp = pt.run(scene, &film, std::atoi(argv[3]), std::atoi(argv[4]), on_pass);
    }
    double sum = 0.0;
    for (int i = 0; i < 3 * film.width() * film.height(); ++i) sum += film.data()[i];
    std::printf("passes %d spp %d sum %.9g\n", passes, spp, sum);
  } catch (const xyzgpu::Error &e) {
    std::fprintf(stderr, "xyzgpu error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
