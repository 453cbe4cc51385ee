// C++ host layer over the xyzgpu C ABI with the shape of the reference
// renderer's own interface, so that code written against xyz::Scene,
// xyz::ThinLensCamera, xyz::ImageFilm and xyz::PathTracer ports by renaming
// the namespace:
//   Scene::Load / Build / FindIntersection / GetWidth / GetHeight /
//   SetDimension / ThinLensCamera / GetLightArea     xyz/core/scene.hpp:39-275
//   ThinLensCamera::MoveTo / MoveBy / LookAt / LookBy  xyz/core/thinlenscamera.cpp:54-69
//   ImageFilm::Save (.pfm raw XYZ, .float CCIR 601 RGB) xyz/core/imagefilm.cpp:90-206
//   PathTracer::run (spp loop, periodic save)          xyz/integrator/integrator.cpp:88-162
// Differences: the scene is loaded from arrays (the MQO parser is not part of
// the hot path), FindIntersection and the estimator work on batches of rays
// and pixels on the GPU, and failures throw xyzgpu::Error carrying the ABI's
// code and message (the reference prints to stderr and carries on).
// Header-only; link with libxyzgpu.so.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "xyzgpu.h"

namespace xyzgpu {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != XYZGPU_OK) throw Error(rc, xyzgpu_last_error());
}

// Thin-lens camera with the reference's defaults (xyz/core/thinlenscamera.cpp:
// 20-28): eye (0, 1, 4) looking at (0, 1, 0), 25 mm film, f = 35 mm, F1.4.
class ThinLensCamera {
 public:
  ThinLensCamera() {
    c_.eye[0] = 0.0f, c_.eye[1] = 1.0f, c_.eye[2] = 4.0f;
    c_.at[0] = 0.0f, c_.at[1] = 1.0f, c_.at[2] = 0.0f;
    c_.film_size = 0.025f;
    c_.focal_length = 0.035f;
    c_.f_number = 1.4f;
    c_.pinhole = 0;
  }
  void MoveTo(float x, float y, float z) { c_.eye[0] = x, c_.eye[1] = y, c_.eye[2] = z; }
  void MoveBy(float x, float y, float z) { c_.eye[0] += x, c_.eye[1] += y, c_.eye[2] += z; }
  void LookAt(float x, float y, float z) { c_.at[0] = x, c_.at[1] = y, c_.at[2] = z; }
  void LookBy(float x, float y, float z) { c_.at[0] += x, c_.at[1] += y, c_.at[2] += z; }
  void SetFilmSize(float meters) { c_.film_size = meters; }
  void SetFocalLength(float meters) { c_.focal_length = meters; }
  void SetFNumber(float f) { c_.f_number = f; }
  // CONFIG_PINHOLE_CAMERA_MODEL of the reference, chosen at run time here.
  void SetPinhole(bool on) { c_.pinhole = on ? 1 : 0; }
  const xyzgpu_camera &desc() const { return c_; }

 private:
  xyzgpu_camera c_;
};

// Film of W x H CIE XYZ sums (xyz/core/imagefilm.hpp:5-52); pixel (x, y) is
// element y * W + x, row 0 at the bottom.
class ImageFilm {
 public:
  ImageFilm() = default;
  ImageFilm(int width, int height) { Resize(width, height); }
  void Resize(int width, int height) {
    w_ = width;
    h_ = height;
    m_.assign(3 * static_cast<size_t>(width) * height, 0.0f);
  }
  void Clear() { std::fill(m_.begin(), m_.end(), 0.0f); }
  int width() const { return w_; }
  int height() const { return h_; }
  float *data() { return m_.data(); }
  const float *data() const { return m_.data(); }

  // ".pfm": raw XYZ / spp, non-finite pixels written as 0
  // (ImageFilm::SaveAsPfm, imagefilm.cpp:153-206); ".float": CCIR 601-1 RGB /
  // spp with negatives clamped to 0 (ImageFilm::SaveAsFloat, :108-151);
  // ".hdr": Radiance RGBE (ImageFilm::SaveAsHdr, imagefilm_hdr.cpp:124-183,
  // pixels encoded on the GPU); ".bmp": the float2bmp tool's film tone map of
  // XYZ / spp (float2bmp/main.cpp, on the GPU).
  bool Save(const std::string &filename, float spp) const {
    auto ends = [&](const char *sfx) {
      size_t const n = std::char_traits<char>::length(sfx);
      return filename.size() >= n && filename.compare(filename.size() - n, n, sfx) == 0;
    };
    if (ends(".pfm")) return SaveAsPfm(filename, spp);
    if (ends(".float")) return SaveAsFloat(filename, spp);
    if (ends(".hdr")) return xyzgpu_film_save_hdr(filename.c_str(), m_.data(), w_, h_, spp, 0) == XYZGPU_OK;
    if (ends(".bmp")) {
      xyzgpu_tonemap_params tp;
      xyzgpu_tonemap_params_default(&tp);
      tp.scale = 1.0f / spp;
      return xyzgpu_film_save_bmp(filename.c_str(), m_.data(), w_, h_, &tp) == XYZGPU_OK;
    }
    return false;
  }

  // Resumable checkpoint: the sums, the samples done and the parameters that
  // made them (xyzgpu_checkpoint_save / _load).
  bool SaveCheckpoint(const std::string &filename, const xyzgpu_render_params &rp, int spp_done) const {
    return xyzgpu_checkpoint_save(filename.c_str(), &rp, spp_done, m_.data()) == XYZGPU_OK;
  }
  bool LoadCheckpoint(const std::string &filename, xyzgpu_render_params *rp, int *spp_done) {
    if (xyzgpu_checkpoint_load(filename.c_str(), rp, spp_done, nullptr) != XYZGPU_OK) return false;
    Resize(rp->width, rp->height);
    return xyzgpu_checkpoint_load(filename.c_str(), rp, spp_done, m_.data()) == XYZGPU_OK;
  }

 private:
  bool SaveAsPfm(const std::string &filename, float spp) const {
    FILE *f = std::fopen(filename.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "PF\n%d %d\n-1\n", w_, h_);
    float const s = 1.0f / spp;
    for (size_t p = 0; p < m_.size() / 3; ++p) {
      float v[3] = {m_[3 * p] * s, m_[3 * p + 1] * s, m_[3 * p + 2] * s};
      if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2])) v[0] = v[1] = v[2] = 0.0f;
      std::fwrite(v, sizeof(float), 3, f);
    }
    return std::fclose(f) == 0;
  }
  bool SaveAsFloat(const std::string &filename, float spp) const {
    FILE *f = std::fopen(filename.c_str(), "wb");
    if (!f) return false;
    float const s = 1.0f / spp;
    for (size_t p = 0; p < m_.size() / 3; ++p) {
      float const x = m_[3 * p] * s, y = m_[3 * p + 1] * s, z = m_[3 * p + 2] * s;
      // CCIR601_1_XYZ2RGB (libhi/hi/image/color_space.hpp:69-79)
      float rgb[3] = {1.9104f * x - 0.5338f * y - 0.2891f * z, -0.9844f * x + 1.9985f * y - 0.0279f * z,
                      0.0585f * x - 0.1187f * y + 0.9017f * z};
      for (float &c : rgb)
        if (c < 0) c = 0;
      std::fwrite(rgb, sizeof(float), 3, f);
    }
    return std::fclose(f) == 0;
  }
  int w_ = 0, h_ = 0;
  std::vector<float> m_;
};

// The scene: triangles, Lambert / light materials, one light power and a kd-tree
// on the current CUDA device.
class Scene {
 public:
  Scene() { xyzgpu_build_params_default(&bp_); }
  ~Scene() { Clear(); }
  Scene(const Scene &) = delete;
  Scene &operator=(const Scene &) = delete;

  void Clear() {
    if (h_) xyzgpu_scene_destroy(h_);
    h_ = nullptr;
  }

  // Replaces Scene::Load's MQO parsing: the same lists, given as arrays.
  void Load(std::vector<float> positions, std::vector<int32_t> triangles, std::vector<int32_t> tri_material,
            std::vector<float> albedo_xyz, std::vector<int32_t> is_light, const float light_power_xyz[3],
            std::vector<float> normals = {}) {
    Clear();
    pos_ = std::move(positions);
    tri_ = std::move(triangles);
    mat_ = std::move(tri_material);
    alb_ = std::move(albedo_xyz);
    lit_ = std::move(is_light);
    nrm_ = std::move(normals);
    for (int k = 0; k < 3; ++k) power_[k] = light_power_xyz[k];
  }

  xyzgpu_build_params &BuildParams() { return bp_; }

  // Scene::Build (xyz/core/scene.cpp:35): uploads and builds the kd-tree.
  void Build() {
    Clear();
    xyzgpu_scene_desc d{};
    d.positions = pos_.data();
    d.normals = nrm_.empty() ? nullptr : nrm_.data();
    d.n_vertices = static_cast<int>(pos_.size() / 3);
    d.triangles = tri_.data();
    d.tri_material = mat_.data();
    d.n_triangles = static_cast<int>(tri_.size() / 3);
    d.albedo_xyz = alb_.data();
    d.is_light = lit_.data();
    d.n_materials = static_cast<int>(lit_.size());
    for (int k = 0; k < 3; ++k) d.light_power_xyz[k] = power_[k];
    check(xyzgpu_scene_create(&d, &bp_, &h_));
  }

  // Batch Scene::FindIntersection: device rays (8 floats each) -> device hits.
  void FindIntersection(const float *rays, int n, float *hits, void *stream = nullptr) const {
    check(xyzgpu_trace_closest(handle(), rays, n, hits, stream));
  }

  void SetDimension(int width, int height) {
    width_ = width;
    height_ = height;
  }
  int GetWidth() const { return width_; }
  int GetHeight() const { return height_; }
  class ThinLensCamera &ThinLensCamera() { return camera_; }
  const class ThinLensCamera &ThinLensCamera() const { return camera_; }

  float GetLightArea() const {
    xyzgpu_scene_stats st;
    check(xyzgpu_scene_stats_get(handle(), &st));
    return st.light_area;
  }

  // The render parameters of EvalutePathTracing's call (host film, added to).
  xyzgpu_render_params Params(int first_sample, int spp, uint64_t seed, int max_depth = 15, int rr_start_depth = 1,
                              float rr_threshold = 0.2f) const {
    xyzgpu_render_params rp;
    xyzgpu_render_params_default(&rp);
    rp.width = width_;
    rp.height = height_;
    rp.spp = spp;
    rp.spp_offset = first_sample;
    rp.max_depth = max_depth;
    rp.rr_start_depth = rr_start_depth;
    rp.rr_threshold = rr_threshold;
    rp.seed = seed;
    rp.film_location = XYZGPU_FILM_HOST;
    rp.accumulate = 1;
    return rp;
  }

  // Scene::EvalutePathTracing for every pixel and `spp` samples starting at
  // sample index `first_sample`, added to `film` (host memory).
  void EvalutePathTracing(ImageFilm *film, int first_sample, int spp, uint64_t seed, int max_depth = 15,
                          int rr_start_depth = 1, float rr_threshold = 0.2f) const {
    xyzgpu_render_params const rp = Params(first_sample, spp, seed, max_depth, rr_start_depth, rr_threshold);
    if (film->width() != width_ || film->height() != height_) film->Resize(width_, height_);
    check(xyzgpu_render(handle(), &camera_.desc(), &rp, film->data(), nullptr));
  }

  xyzgpu_scene handle() const {
    if (!h_) throw Error(XYZGPU_E_INVALID, "scene is not built");
    return h_;
  }

 private:
  xyzgpu_scene h_ = nullptr;
  xyzgpu_build_params bp_;
  std::vector<float> pos_, alb_, nrm_;
  std::vector<int32_t> tri_, mat_, lit_;
  float power_[3] = {0, 0, 0};
  int width_ = 720, height_ = 480;  // Scene::Scene's SetDimension(720, 480)
  class ThinLensCamera camera_;
};

// PathTracer::run (xyz/integrator/integrator.cpp:88-162): sample passes over
// the whole image, `interval` samples per pass; after each pass the callback
// receives the film and the number of samples so far (the reference saves a
// .pfm there) and may return false to stop.
class PathTracer {
 public:
  int max_depth = 15;
  int rr_start_depth = 1;
  float rr_threshold = 0.2f;
  uint64_t seed = 0;

  // checkpoint: if not empty, the film, the samples done and the parameters
  // are saved there after every pass (xyzgpu_checkpoint_save), and run()
  // starts from that file when it exists and matches this render (same image
  // size, seed, depth and roulette), so a stopped render continues where it
  // stopped with the film it would have had.
  std::string checkpoint;

  int run(const Scene &scene, ImageFilm *film, int total_spp, int interval,
          const std::function<bool(const ImageFilm &, int)> &on_pass = {}) const {
    film->Resize(scene.GetWidth(), scene.GetHeight());
    int done = 0;
    if (!checkpoint.empty()) {
      xyzgpu_render_params saved;
      int saved_done = 0;
      ImageFilm loaded;
      xyzgpu_render_params const want = scene.Params(0, 0, seed, max_depth, rr_start_depth, rr_threshold);
      if (loaded.LoadCheckpoint(checkpoint, &saved, &saved_done) && saved.width == want.width &&
          saved.height == want.height && saved.seed == want.seed && saved.max_depth == want.max_depth &&
          saved.rr_start_depth == want.rr_start_depth && saved.rr_threshold == want.rr_threshold &&
          saved_done <= total_spp) {
        *film = std::move(loaded);
        done = saved_done;
      }
    }
    while (done < total_spp) {
      int const n = std::min(interval, total_spp - done);
      scene.EvalutePathTracing(film, done, n, seed, max_depth, rr_start_depth, rr_threshold);
      done += n;
      if (!checkpoint.empty() &&
          !film->SaveCheckpoint(checkpoint, scene.Params(0, done, seed, max_depth, rr_start_depth, rr_threshold),
                                done))
        throw Error(XYZGPU_E_INVALID, "PathTracer: cannot write checkpoint " + checkpoint);
      if (on_pass && !on_pass(*film, done)) break;
    }
    return done;
  }
};

// PathTracer::run with the learned path guide (xyzgpu_guide_*, no
// counterpart in the reference): the first `train_fraction` of the samples
// train the guide (Adam steps after every pass) and, drawn while the guide is
// still immature, go to a scratch film; the rest are rendered with the guide
// into `film`, so `film` holds total_spp - training samples, the number run()
// returns and the callback receives.  The estimator is unbiased with any
// guide (one-sample MIS with Lambert sampling).
class GuidedPathTracer {
 public:
  int max_depth = 15;
  int rr_start_depth = 1;
  float rr_threshold = 0.2f;
  uint64_t seed = 0;
  double train_fraction = 0.25;
  xyzgpu_guide_config config;

  GuidedPathTracer() { xyzgpu_guide_config_default(&config); }

  int run(const Scene &scene, ImageFilm *film, int total_spp, int interval,
          const std::function<bool(const ImageFilm &, int)> &on_pass = {}) const {
    film->Resize(scene.GetWidth(), scene.GetHeight());
    ImageFilm scratch(scene.GetWidth(), scene.GetHeight());
    xyzgpu_guide g = nullptr;
    check(xyzgpu_guide_create(scene.handle(), &config, &g));
    struct Guard {
      xyzgpu_guide g;
      ~Guard() { xyzgpu_guide_destroy(g); }
    } guard{g};
    int const train = std::min(total_spp, static_cast<int>(total_spp * train_fraction));
    int done = 0;
    while (done < total_spp) {
      bool const training = done < train;
      int const n = std::min(interval, (training ? train : total_spp) - done);
      xyzgpu_render_params rp;
      xyzgpu_render_params_default(&rp);
      rp.width = scene.GetWidth();
      rp.height = scene.GetHeight();
      rp.spp = n;
      rp.spp_offset = done;
      rp.max_depth = max_depth;
      rp.rr_start_depth = rr_start_depth;
      rp.rr_threshold = rr_threshold;
      rp.seed = seed;
      rp.film_location = XYZGPU_FILM_HOST;
      rp.accumulate = 1;
      check(xyzgpu_render_guided(g, &scene.ThinLensCamera().desc(), &rp, training ? 1 : 0,
                                 training ? scratch.data() : film->data(), nullptr));
      done += n;
      if (!training && on_pass && !on_pass(*film, done - train)) break;
    }
    return done - train;
  }
};

}  // namespace xyzgpu
