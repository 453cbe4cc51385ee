// C harness around the reference renderer's own path tracer, compiled from the
// reference sources where they lie (recipe: oracle/Makefile, output only under
// oracle/_ref/).  TEST INFRASTRUCTURE: only tests/, the smoke check and
// bench.py's CPU legs load the library built from this file.
//
// The reference drives `xyz::Scene` from its MQO loader and a GUI shell; the
// harness fills the same members directly so that triangle ids are the caller's
// ids (xyz/core/scene_mqo.cpp:676-692 would Morton-sort them) and calls:
//   * Scene::Build                 xyz/core/scene.cpp:35 -> KDTree::Build
//   * Scene::FindIntersection      xyz/core/scene.hpp:277-295
//   * Scene::EvalutePathTracing    xyz/core/scene_pathtracing.cpp:11-144
// with the pixel loop of PathTracer::run (xyz/integrator/integrator.cpp:119-128).
// Random numbers come from the Philox stream of oracle/philox.h through the
// reference's IPrimarySample interface (xyz/bsdf/bsdf.hpp:10-14) instead of the
// single global mt19937_64 (integrator.cpp:12-25), so that each (pixel, sample)
// path reads a fixed stream that other implementations can reproduce.
#include <atomic>
#include <fstream>
#include <vector>
#include <unordered_map>

#define private public
#define protected public
#include <core/scene.hpp>
#undef private
#undef protected
#include <bsdf/bsdf.hpp>
#include <bsdf/lambert.hpp>
#include <bsdf/light.hpp>
#include <bsdf/metal.hpp>
#include <bsdf/mirror.hpp>
#include <geom/intersection.hpp>
#include <geom/triangle.hpp>

extern "C" {
#include "philox.h"
}

std::size_t xyzref_kmax = 16;         // xyz/core/config.hpp:30
float xyzref_rr_threshold = 0.2f;     // xyz/core/config.hpp:60

namespace {

class PhiloxSample : public xyz::IPrimarySample {
 public:
  PhiloxSample(std::uint64_t seed, std::uint32_t pixel, std::uint32_t sample) {
    xyzo_stream_init(&s_, seed, pixel, sample, 0u);
  }
  virtual xyz::float_t next() { return xyzo_stream_next(&s_); }
  std::uint32_t dims() const { return s_.dim; }

 private:
  xyzo_stream s_;
};

struct Harness {
  std::unordered_map<xyz::Triangle const *, int> ids;
  int width = 0, height = 0;
};

Harness &H() {
  static Harness h;
  return h;
}

void ClearScene() {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  scene.Clear();
  H().ids.clear();
}

// Runs body(i) for i in [lo, hi) on `nthreads` std::threads pulling chunks of
// `chunk` indices from a shared counter (nthreads <= 0: hardware concurrency).
template <class F>
void ParallelFor(int lo, int hi, int chunk, int nthreads, F const &body) {
  if (nthreads <= 0) {
    nthreads = static_cast<int>(std::thread::hardware_concurrency());
    if (nthreads <= 0) nthreads = 1;
  }
  std::atomic<int> next(lo);
  auto worker = [&]() {
    for (;;) {
      int const b = next.fetch_add(chunk);
      if (b >= hi) break;
      int const e = std::min(hi, b + chunk);
      for (int i = b; i < e; ++i) body(i);
    }
  };
  if (nthreads == 1) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}

}  // namespace

extern "C" {

int xyzref_is_pinhole(void) {
#ifdef CONFIG_PINHOLE_CAMERA_MODEL
  return 1;
#else
  return 0;
#endif
}

// Light power Φ as CIE XYZ: the Mercury-arc SPD through the reference's CMF
// (xyz/core/config.hpp:81-95).  The estimator is linear in it per channel.
void xyzref_light_power_xyz(float out[3]) {
  xyz::CIE_XYZ_Color const c = xyz::GetLightPowerXYZ();
  out[0] = c[0];
  out[1] = c[1];
  out[2] = c[2];
}

void xyzref_set_path_params(int kmax, float rr_threshold) {
  xyzref_kmax = static_cast<std::size_t>(kmax);
  xyzref_rr_threshold = rr_threshold;
}

// Kinds of the next scene's non-light materials: 0 Lambert (default),
// 2 Mirror (xyz/bsdf/mirror.cpp), 3 Metal with its shininess
// (xyz/bsdf/metal.cpp, Metal(shininess, albedo)).  Consumed by the next
// xyzref_scene_create.
static std::vector<int> g_kind;
static std::vector<float> g_shininess;
void xyzref_material_kinds(int nm, const int *kind, const float *shininess) {
  g_kind.assign(kind, kind + nm);
  g_shininess.assign(shininess, shininess + nm);
}

// Builds the scene.  Vertices `pos` (3*nv floats), optional per-vertex shading
// normals `nrm` (3*nv or NULL), triangles `tri` (3*nt ints) with material ids
// `tri_mat`; materials carry an XYZ albedo and a light flag.  Lights are
// accumulated into the area CDF in triangle order, as xyz/core/scene_mqo.cpp:
// 512-519 does.  Returns the number of light triangles, or -1 on bad input.
int xyzref_scene_create(int nv, const float *pos, const float *nrm, int nt,
                        const int *tri, const int *tri_mat, int nm,
                        const float *mat_albedo_xyz, const int *mat_is_light,
                        int kd_max_bucket, int kd_max_depth) {
  ClearScene();
  xyz::Scene &scene = xyz::Scene::GetInstance();
  for (int m = 0; m < nm; ++m) {
    int const kind = m < static_cast<int>(g_kind.size()) ? g_kind[m] : 0;
    xyz::float3_t const alb(mat_albedo_xyz[3 * m + 0], mat_albedo_xyz[3 * m + 1], mat_albedo_xyz[3 * m + 2]);
    if (mat_is_light[m]) {
      scene.bsdfs_.push_back(new xyz::Light());
    } else if (kind == 2) {
      scene.bsdfs_.push_back(new xyz::Mirror());
    } else if (kind == 3) {
      scene.bsdfs_.push_back(new xyz::Metal(g_shininess[m], alb));
    } else {
      scene.bsdfs_.push_back(new xyz::Lambert(xyz::float3_t(
          mat_albedo_xyz[3 * m + 0], mat_albedo_xyz[3 * m + 1],
          mat_albedo_xyz[3 * m + 2])));
    }
  }
  int nlights = 0;
  for (int i = 0; i < nt; ++i) {
    int const a = tri[3 * i + 0], b = tri[3 * i + 1], c = tri[3 * i + 2];
    int const m = tri_mat[i];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv || m < 0 ||
        m >= nm) {
      ClearScene();
      return -1;
    }
    xyz::float3_t const p0(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
    xyz::float3_t const p1(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
    xyz::float3_t const p2(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
    xyz::Triangle *t;
    if (nrm) {
      xyz::float3_t const n0(nrm[3 * a], nrm[3 * a + 1], nrm[3 * a + 2]);
      xyz::float3_t const n1(nrm[3 * b], nrm[3 * b + 1], nrm[3 * b + 2]);
      xyz::float3_t const n2(nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]);
      t = new xyz::Triangle(m, p0, p1, p2, n0, n1, n2, 0, 0, 1, 0, 0, 1);
    } else {
      t = new xyz::Triangle(m, p0, p1, p2, 0, 0, 1, 0, 0, 1);
    }
    scene.triangles_.push_back(t);
    H().ids[t] = i;
    scene.rSurfaceArea_ += t->area();
    if (mat_is_light[m]) {
      scene.lights_.push_back(t);
      scene.lightsCdf_.push_back(scene.lightsCdf_.back() + t->area());
      ++nlights;
    }
  }
  g_kind.clear();
  g_shininess.clear();
  scene.kdtree_.SetMaxBucketSize(static_cast<std::size_t>(kd_max_bucket));
  scene.kdtree_.SetMaxHierarchyDepth(static_cast<std::size_t>(kd_max_depth));
  scene.Build();
  return nlights;
}

void xyzref_scene_destroy(void) { ClearScene(); }

float xyzref_light_area(void) {
  return xyz::Scene::GetInstance().GetLightArea();
}

// Camera as the reference models it (xyz/core/thinlenscamera.cpp:20-28,71-90):
// eye, gaze point, film size, focal length and F-number; up is +y.
void xyzref_set_camera(const float eye[3], const float at[3], float film_size,
                       float focal_length, float f_number, int width,
                       int height) {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  xyz::ThinLensCamera &cam = scene.camera_;
  cam.vPrincipalPoint_ = xyz::float3_t(eye[0], eye[1], eye[2]);
  cam.vGazingPoint_ = xyz::float3_t(at[0], at[1], at[2]);
  cam.fFilmSize_ = film_size;
  cam.fFocalLength_ = focal_length;
  cam.fFNumber_ = f_number;
  scene.SetDimension(width, height);
  cam.Reset();
  H().width = width;
  H().height = height;
}

// Closest hit for n rays (KDTree traversal + double-faced Möller-Trumbore).
// tri_out = triangle id or -1; t/f/g/back as the reference's Intersection.
void xyzref_trace(int n, const float *org, const float *dir, int *tri_out,
                  float *t_out, float *f_out, float *g_out, int *back_out,
                  int nthreads) {
  xyz::Scene const &scene = xyz::Scene::GetInstance();
  ParallelFor(0, n, 256, nthreads, [&](int i) {
    xyz::Intersection param;
    xyz::float3_t const o(org[3 * i], org[3 * i + 1], org[3 * i + 2]);
    xyz::float3_t const d(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    xyz::Triangle const *t = scene.kdtree_.FindIntersection(o, d, &param);
    if (t) {
      tri_out[i] = H().ids.at(t);
      t_out[i] = param.t_max();
      f_out[i] = param.f();
      g_out[i] = param.g();
      back_out[i] = param.is_back_side() ? 1 : 0;
    } else {
      tri_out[i] = -1;
      t_out[i] = 0;
      f_out[i] = 0;
      g_out[i] = 0;
      back_out[i] = 0;
    }
  });
}

// One path sample (pixel px,py, sample s): the XYZ estimate and the number of
// random dimensions the reference consumed.
int xyzref_eval_path(int px, int py, int s, std::uint64_t seed, float out[3]) {
  xyz::Scene const &scene = xyz::Scene::GetInstance();
  int const W = H().width, Hh = H().height;
  PhiloxSample sample(seed, static_cast<std::uint32_t>(py * W + px),
                      static_cast<std::uint32_t>(s));
  xyz::float_t const jx = sample.next();
  xyz::float_t const jy = sample.next();
  xyz::CIE_XYZ_Color color;
  scene.EvalutePathTracing((px + jx) / W, (py + jy) / Hh, &color, sample);
  out[0] = color[0];
  out[1] = color[1];
  out[2] = color[2];
  return static_cast<int>(sample.dims());
}

// Film accumulation of PathTracer::run for samples [s0, s0+spp) over pixel rows
// [y0, y1): film[y*W+x] += color per sample, in sample order.  film is W*H*3,
// not divided by spp.  Rows are shared out over `nthreads` threads (a row
// belongs to one thread, so film updates do not race), as the reference's
// disabled row-parallel loop intends (xyz/integrator/integrator.cpp:120).
void xyzref_render(int s0, int spp, std::uint64_t seed, int y0, int y1,
                   float *film, int nthreads) {
  xyz::Scene const &scene = xyz::Scene::GetInstance();
  int const W = H().width, Hh = H().height;
  for (int s = s0; s < s0 + spp; ++s) {
    ParallelFor(y0, y1, 1, nthreads, [&](int y) {
      for (int x = 0; x < W; ++x) {
        PhiloxSample sample(seed, static_cast<std::uint32_t>(y * W + x),
                            static_cast<std::uint32_t>(s));
        xyz::float_t const jx = sample.next();
        xyz::float_t const jy = sample.next();
        xyz::CIE_XYZ_Color color;
        scene.EvalutePathTracing((x + jx) / W, (y + jy) / Hh, &color, sample);
        float *f = film + 3 * (static_cast<std::size_t>(y) * W + x);
        f[0] += color[0];
        f[1] += color[1];
        f[2] += color[2];
      }
    });
  }
}

}  // extern "C"

// Triangle's stored vectors are private: an explicit instantiation may name
// private members and hands their pointers out.
namespace {
template <int K>
struct TriMember {
  typedef xyz::Triangle::float3_t const xyz::Triangle::*type;
  friend type tri_member(TriMember);
};
template <typename Tag, typename Tag::type M>
struct ExposeTri {
  friend typename Tag::type tri_member(Tag) { return M; }
};
template struct ExposeTri<TriMember<0>, &xyz::Triangle::v0_>;
template struct ExposeTri<TriMember<1>, &xyz::Triangle::e1_>;
template struct ExposeTri<TriMember<2>, &xyz::Triangle::e2_>;
template struct ExposeTri<TriMember<3>, &xyz::Triangle::ng_>;
template struct ExposeTri<TriMember<4>, &xyz::Triangle::n0_>;
template struct ExposeTri<TriMember<5>, &xyz::Triangle::s1_>;
template struct ExposeTri<TriMember<6>, &xyz::Triangle::s2_>;
}  // namespace

extern "C" {

// ---- The reference's MQO loader (Scene::Load, xyz/core/scene_mqo.cpp:547-696)
// on a file: the triangles in the order it leaves them (Morton-sorted), their
// stored geometry (v0, e1, e2, geometric normal, shading n0, s1, s2), materials
// and the camera the file's Scene chunk sets.  Returns the triangle count.
int xyzref_load_mqo(const char *path) {
  ClearScene();
  std::ifstream in(path);
  if (!in) return -1;
  xyz::Scene &scene = xyz::Scene::GetInstance();
  scene.Load(in);
  return static_cast<int>(scene.triangles_.size());
}

void xyzref_mqo_counts(int *n_tris, int *n_mats, int *n_lights) {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  *n_tris = static_cast<int>(scene.triangles_.size());
  *n_mats = static_cast<int>(scene.bsdfs_.size());
  *n_lights = static_cast<int>(scene.lights_.size());
}

// geo: 21 floats per triangle (v0, e1, e2, ng, n0, s1, s2); mat: material id
void xyzref_mqo_triangles(float *geo, int *mat) {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  for (std::size_t i = 0; i < scene.triangles_.size(); ++i) {
    xyz::Triangle const *t = scene.triangles_[i];
    xyz::float3_t const v[7] = {t->*tri_member(TriMember<0>()), t->*tri_member(TriMember<1>()),
                                t->*tri_member(TriMember<2>()), t->*tri_member(TriMember<3>()),
                                t->*tri_member(TriMember<4>()), t->*tri_member(TriMember<5>()),
                                t->*tri_member(TriMember<6>())};
    for (int k = 0; k < 7; ++k)
      for (int c = 0; c < 3; ++c) geo[21 * i + 3 * k + c] = v[k][c];
    mat[i] = static_cast<int>(t->bsdf());
  }
}

// kind: Bsdf::What() (0 Lambert, 1 mirror, 2 glass, 3 metal, 4 light);
// albedo: Lambert / metal XYZ; shininess: metal exponent
void xyzref_mqo_materials(int *kind, float *albedo, float *shininess) {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  for (std::size_t m = 0; m < scene.bsdfs_.size(); ++m) {
    xyz::Bsdf const *b = scene.bsdfs_[m];
    kind[m] = static_cast<int>(b->What());
    albedo[3 * m] = albedo[3 * m + 1] = albedo[3 * m + 2] = 0.0f;
    shininess[m] = 0.0f;
    if (b->What() == xyz::Bsdf::LAMBERT) {
      xyz::float3_t const a = static_cast<xyz::Lambert const *>(b)->albedo();
      for (int c = 0; c < 3; ++c) albedo[3 * m + c] = a[c];
    } else if (b->What() == xyz::Bsdf::METAL) {
      xyz::Metal const *mt = static_cast<xyz::Metal const *>(b);
      for (int c = 0; c < 3; ++c) albedo[3 * m + c] = mt->albedo()[c];
      shininess[m] = mt->sininess();
    }
  }
}

void xyzref_mqo_camera(float eye[3], float at[3]) {
  xyz::Scene &scene = xyz::Scene::GetInstance();
  xyz::float3_t const e = scene.ThinLensCamera().Eye(), a = scene.ThinLensCamera().At();
  for (int c = 0; c < 3; ++c) {
    eye[c] = e[c];
    at[c] = a[c];
  }
}

// The named spectra of libhi/hi/image/spectrum.cpp:170-476 (lights, then the
// Macbeth colour checker), in the order listed by xyzref_spectrum_names.
const char *xyzref_spectrum_names(void) {
  return "LightSourceA LightSourceB LightSourceC LightD65 LightD100 LightStandardWarmWhite LightWhite LightStandardWhite LightDaylight LightWarmWhiteDeLuxe LightSoftWhite LightCoolWhiteDeLuxe LightMercuryArcLamp MccDarkSkin MccLightSkin MccBlueSky MccFoliage MccBlueFlower MccBluishGreen MccOrange MccPurplishBlue MccModerateRed MccPurple MccYellowGreen MccOrangeYellow MccBlue MccGreen MccRed MccYellow MccMagenta MccCyan MccWhite MccNeutral80 MccNeutral65 MccNeutral50 MccNeutral35 MccBlack";
}

int xyzref_named_spectrum(int id, float out[31]) {
  hi::basic_spectrum const *s = nullptr;
  switch (id) {
    case 0: s = &hi::basic_spectrum::LightSourceA(); break;
    case 1: s = &hi::basic_spectrum::LightSourceB(); break;
    case 2: s = &hi::basic_spectrum::LightSourceC(); break;
    case 3: s = &hi::basic_spectrum::LightD65(); break;
    case 4: s = &hi::basic_spectrum::LightD100(); break;
    case 5: s = &hi::basic_spectrum::LightStandardWarmWhite(); break;
    case 6: s = &hi::basic_spectrum::LightWhite(); break;
    case 7: s = &hi::basic_spectrum::LightStandardWhite(); break;
    case 8: s = &hi::basic_spectrum::LightDaylight(); break;
    case 9: s = &hi::basic_spectrum::LightWarmWhiteDeLuxe(); break;
    case 10: s = &hi::basic_spectrum::LightSoftWhite(); break;
    case 11: s = &hi::basic_spectrum::LightCoolWhiteDeLuxe(); break;
    case 12: s = &hi::basic_spectrum::LightMercuryArcLamp(); break;
    case 13: s = &hi::basic_spectrum::MccDarkSkin(); break;
    case 14: s = &hi::basic_spectrum::MccLightSkin(); break;
    case 15: s = &hi::basic_spectrum::MccBlueSky(); break;
    case 16: s = &hi::basic_spectrum::MccFoliage(); break;
    case 17: s = &hi::basic_spectrum::MccBlueFlower(); break;
    case 18: s = &hi::basic_spectrum::MccBluishGreen(); break;
    case 19: s = &hi::basic_spectrum::MccOrange(); break;
    case 20: s = &hi::basic_spectrum::MccPurplishBlue(); break;
    case 21: s = &hi::basic_spectrum::MccModerateRed(); break;
    case 22: s = &hi::basic_spectrum::MccPurple(); break;
    case 23: s = &hi::basic_spectrum::MccYellowGreen(); break;
    case 24: s = &hi::basic_spectrum::MccOrangeYellow(); break;
    case 25: s = &hi::basic_spectrum::MccBlue(); break;
    case 26: s = &hi::basic_spectrum::MccGreen(); break;
    case 27: s = &hi::basic_spectrum::MccRed(); break;
    case 28: s = &hi::basic_spectrum::MccYellow(); break;
    case 29: s = &hi::basic_spectrum::MccMagenta(); break;
    case 30: s = &hi::basic_spectrum::MccCyan(); break;
    case 31: s = &hi::basic_spectrum::MccWhite(); break;
    case 32: s = &hi::basic_spectrum::MccNeutral80(); break;
    case 33: s = &hi::basic_spectrum::MccNeutral65(); break;
    case 34: s = &hi::basic_spectrum::MccNeutral50(); break;
    case 35: s = &hi::basic_spectrum::MccNeutral35(); break;
    case 36: s = &hi::basic_spectrum::MccBlack(); break;
    default: return -1;
  }
  for (int i = 0; i < 31; ++i) out[i] = (*s)[i];
  return 0;
}

int xyzref_max_threads(void) {
  int const n = static_cast<int>(std::thread::hardware_concurrency());
  return n > 0 ? n : 1;
}

}  // extern "C"
