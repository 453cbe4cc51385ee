// C harness around the reference's spectral renderer (renderer/, namespace
// tgir), compiled from its sources by oracle/Makefile into oracle/_ref/.
// TEST INFRASTRUCTURE: only tests/ load it.
//
// It fills tgir::Scene from arrays (31-bin albedo spectra per material) and
// calls tgir::Scene::EvaluteRussianRoulette (renderer/core/SceneStrategy.cpp:
// 11-149): one wavelength bin per path, next-event estimation before the
// depth cap, Russian roulette on the scalar spectral throughput, XYZ out via
// hi::spd2xyz(bin, L) (libhi/hi/image/spectrum.cpp:561-567).  Each row of
// each sample pass draws from its own std::mt19937_64 (the reference's Ptrr
// driver keeps one generator per thread, renderer/sampler/Ptrr.cpp:24), so the
// comparison with other implementations is statistical.
#include <unordered_map>

#define private public
#define protected public
#include <core/Scene.hpp>
#undef private
#undef protected
#include <bsdf/Bsdf.hpp>
#include <bsdf/Lambert.hpp>
#include <bsdf/Light.hpp>
#include <geom/Intersection.hpp>
#include <geom/Triangle.hpp>

std::size_t xyztwin_kmax = 8;          // renderer/core/config.hpp:34
double xyztwin_rr_threshold = 0.2;

namespace {
template <class F>
void ParallelFor(int lo, int hi, int nthreads, F const &body) {
  if (nthreads <= 0) {
    nthreads = static_cast<int>(std::thread::hardware_concurrency());
    if (nthreads <= 0) nthreads = 1;
  }
  std::atomic<int> next(lo);
  auto worker = [&]() {
    for (;;) {
      int const i = next.fetch_add(1);
      if (i >= hi) break;
      body(i);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}
}  // namespace

extern "C" {

int xyztwin_is_pinhole(void) {
#ifdef CONFIG_PINHOLE_CAMERA_MODEL
  return 1;
#else
  return 0;
#endif
}

void xyztwin_light_spd(float out[31]) {
  tgir::SpectrumData const &s = tgir::GetLightPower();
  for (int i = 0; i < 31; ++i) out[i] = s[i];
}

void xyztwin_set_path_params(int kmax, double rr_threshold) {
  xyztwin_kmax = static_cast<std::size_t>(kmax);
  xyztwin_rr_threshold = rr_threshold;
}

int xyztwin_scene_create(int nv, const float *pos, const float *nrm, int nt, const int *tri,
                         const int *tri_mat, int nm, const float *albedo_spd, const int *is_light) {
  tgir::Scene &scene = tgir::Scene::GetInstance();
  scene.Clear();
  for (int m = 0; m < nm; ++m) {
    if (is_light[m]) {
      scene.bsdfs_.push_back(new tgir::Light());
    } else {
      tgir::SpectrumData a;
      for (int i = 0; i < 31; ++i) a[i] = albedo_spd[31 * m + i];
      scene.bsdfs_.push_back(new tgir::Lambert(a));
    }
  }
  int nl = 0;
  for (int i = 0; i < nt; ++i) {
    int const a = tri[3 * i], b = tri[3 * i + 1], c = tri[3 * i + 2], m = tri_mat[i];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv || m < 0 || m >= nm) {
      scene.Clear();
      return -1;
    }
    tgir::Vector3 const p0(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
    tgir::Vector3 const p1(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
    tgir::Vector3 const p2(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
    tgir::Triangle *t;
    if (nrm) {
      tgir::Vector3 const n0(nrm[3 * a], nrm[3 * a + 1], nrm[3 * a + 2]);
      tgir::Vector3 const n1(nrm[3 * b], nrm[3 * b + 1], nrm[3 * b + 2]);
      tgir::Vector3 const n2(nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]);
      t = new tgir::Triangle(m, p0, p1, p2, n0, n1, n2, 0, 0, 1, 0, 0, 1);
    } else {
      t = new tgir::Triangle(m, p0, p1, p2, 0, 0, 1, 0, 0, 1);
    }
    scene.triangles_.push_back(t);
    if (is_light[m]) {
      scene.lights_.push_back(t);
      scene.lightsCdf_.push_back(scene.lightsCdf_.back() + t->area());
      ++nl;
    }
  }
  scene.Build();
  return nl;
}

void xyztwin_set_camera(const float eye[3], const float at[3], float film_size, float focal_length,
                        float f_number, int width, int height) {
  tgir::Scene &scene = tgir::Scene::GetInstance();
  tgir::Camera &cam = scene.camera_;
  cam.vPrincipalPoint_ = tgir::Vector3(eye[0], eye[1], eye[2]);
  cam.vGazingPoint_ = tgir::Vector3(at[0], at[1], at[2]);
  cam.fFilmSize_ = film_size;
  cam.fFocalLength_ = focal_length;
  cam.fFNumber_ = f_number;
  scene.SetDimension(width, height);
  cam.Reset();
}

// film[y*W+x] += XYZ of each sample in [s0, s0+spp); rows in parallel.
void xyztwin_render(int s0, int spp, unsigned long long seed, float *film, int nthreads) {
  tgir::Scene const &scene = tgir::Scene::GetInstance();
  int const W = scene.GetWidth(), H = scene.GetHeight();
  for (int s = s0; s < s0 + spp; ++s) {
    ParallelFor(0, H, nthreads, [&](int y) {
      std::seed_seq sq{static_cast<unsigned>(seed), static_cast<unsigned>(seed >> 32),
                       static_cast<unsigned>(s), static_cast<unsigned>(y)};
      std::mt19937_64 random(sq);
      for (int x = 0; x < W; ++x) {
        tgir::SpectrumVector c;
        scene.EvaluteRussianRoulette(x, y, c, random);
        float *f = film + 3 * (static_cast<std::size_t>(y) * W + x);
        f[0] += c[0];
        f[1] += c[1];
        f[2] += c[2];
      }
    });
  }
}

}  // extern "C"
