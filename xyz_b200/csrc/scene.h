// Host-side scene object behind the xyzgpu_scene handle, plus the error and
// CUDA-check helpers shared by the C ABI implementation files.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/xyzgpu.h"
#include "common.cuh"
#include "kdtree.h"

namespace xyzgpu {

int set_error(int code, const char *fmt, ...);
void clear_error();

#define XYZ_CUDA_TRY(call)                                                                   \
  do {                                                                                       \
    cudaError_t const e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                                   \
      return ::xyzgpu::set_error(XYZGPU_E_CUDA, "%s failed: %s (%s:%d)", #call,              \
                                 cudaGetErrorString(e_), __FILE__, __LINE__);                \
  } while (0)

// Device buffers of one render wave (paths in flight), kept between calls.
struct RenderWorkspace {
  int64_t capacity = 0;   // paths
  int max_iters = 0;      // count slots allocated
  float4 *beta = nullptr;     // throughput xyz, fSamplingNext
  uint32_t *misc = nullptr;   // dim | k << 16 | specular << 31
  float4 *radiance = nullptr; // accumulated XYZ of the path
  float4 *q_o[2] = {nullptr, nullptr};
  float4 *q_d[2] = {nullptr, nullptr};
  int32_t *q_slot[2] = {nullptr, nullptr};
  float4 *hits = nullptr;
  float4 *s_o = nullptr, *s_d = nullptr, *s_pb = nullptr;
  float4 *s_m = nullptr;        // metal vertices' next-event terms (nk2, nk3, lobe pdf, factor)
  int32_t *s_target = nullptr;
  float *fsn = nullptr;         // spectral modes: fSamplingNext per path
  int32_t *s_slot = nullptr;    // spectral modes: path slot of each shadow ray
  int32_t *counts = nullptr;  // per iteration counters (see render.cu)
  unsigned long long *tally = nullptr;  // [0] ext rays [1] shadow rays [2] visible,
                                        // [8..13] traversal counters of COUNTERS renders,
                                        // [16..] extension / shadow rays per iteration
  int profile_iters = 0;
  std::vector<cudaEvent_t> events;      // timing pairs of TIMING renders
  float *film_dev = nullptr;  // staging film for host-film renders
  float *film_pinned = nullptr;
  int64_t film_elems = 0;
};

struct SceneImpl {
  int device = 0;
  int n_tris = 0, n_lights = 0, n_materials = 0;
  bool smooth = false;
  DevScene dev{};
  // device allocations owned here
  float4 *d_tri = nullptr, *d_ng = nullptr, *d_sn = nullptr, *d_mat = nullptr;
  float *d_emission = nullptr;  // per-material emission scale, ones at creation
  int32_t *d_lights = nullptr;
  float *d_cdf = nullptr;
  float *d_spd = nullptr;  // 31-bin albedo spectra (spectral modes)
  float *d_shininess = nullptr;  // per material
  int n_specular = 0;            // materials of kind mirror or metal
  uint2 *d_nodes = nullptr;
  int32_t *d_refs = nullptr;
  int64_t n_nodes = 0, n_refs = 0, n_leaves = 0, n_empty = 0;
  int depth = 0;
  int64_t device_bytes = 0;
  double build_ms = 0.0;
  RenderWorkspace ws;
  xyzgpu_render_counters counters{};
  xyzgpu_render_profile profile{};
  bool profile_pending = false;  // profile needs the events / counters read back
  int profile_mode = 0;
  std::vector<int> event_class;   // class of each recorded event pair
  int32_t *d_fetch = nullptr;  // work-fetch counters of the trace API kernel
  unsigned long long *d_trace_counts = nullptr;
};

// Wave buffers are shared by every scene on a device (single and batched
// renders): the largest wave asked for so far stays allocated, and renders on
// different streams are ordered by an event so that they never use the buffers
// at the same time.  Hold `mu` while using them.
struct SharedWaves {
  std::mutex mu;
  RenderWorkspace ws;  // only the wave buffers (beta .. counts) are used
  cudaEvent_t done = nullptr;
  cudaStream_t last = nullptr;
};
SharedWaves &shared_waves(int device);
int ensure_wave_buffers(RenderWorkspace &w, int64_t capacity, int iters);
extern const int64_t kBytesPerPath;  // wave buffer bytes per path

// Kernels' host-side launchers (trace.cu, render.cu, kdbuild.cu).
int trace_api_launch(SceneImpl &s, const float *rays, int n, float *hits, cudaStream_t st,
                     xyzgpu_trace_counters *counters);
// Path-replay adjoint of a render (xyzgpu_adjoint): gradients are added to
// g_albedo (3 per material) and g_emission (1 per material).
struct AdjointArgs {
  const float *d_film;  // W * H * 3, device
  float *g_albedo;
  float *g_emission;
};

// Guided render (xyzgpu_render_guided): the guide's per-wave buffers and
// hooks (guide.cu).
struct GuideImpl;
struct GuideWave {
  void *mix = nullptr;       // fp16, 40 per extension-queue entry
  float *records = nullptr;  // training records of the wave (16 floats x train_bounces per path)
  int train_bounces = 0;     // 0: no training records
  float alpha = 0.5f;
  int guide_bounces = 0;     // bounces sampled with the guide
};
struct GuideHooks {
  GuideImpl *g;
  bool train;
};
int guide_wave_prepare(GuideImpl &g, int64_t capacity, bool train, cudaStream_t st, GuideWave *out);
int guide_infer_launch(GuideImpl &g, const float4 *qo, const float4 *qd, const float4 *hits,
                       const int32_t *count, const DevScene &S, void *mix, cudaStream_t st);
int guide_train_on_wave(GuideImpl &g, const float4 *radiance, int64_t npaths, cudaStream_t st);

// Importance-driven render (xyzgpu_render_importon): the light-importance map
// and its per-wave histogram buffer (importon.cu).
struct ImportonImpl;
struct ImportonHooks {
  ImportonImpl *m;
};
int importon_wave_prepare(ImportonImpl &m, int64_t capacity, float **cdf);
int importon_query_launch(ImportonImpl &m, const float4 *qo, const float4 *qd, const float4 *hits,
                          const int32_t *count, const DevScene &S, float *cdf, cudaStream_t st);
int importon_guide_bounces(const ImportonImpl &m);

int render_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp,
                  float *film, cudaStream_t st, const AdjointArgs *adj = nullptr,
                  const GuideHooks *guide = nullptr, const ImportonHooks *imp = nullptr);
// Argument checks of xyzgpu_render (api.cu).
int check_render_args(const char *who, xyzgpu_scene scene, const xyzgpu_camera *cam,
                      const xyzgpu_render_params *rp);
void render_workspace_free(RenderWorkspace &ws);
int render_collect(SceneImpl &s);
int render_noalloc_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp,
                          float *film, cudaStream_t st);
int kd_build_device(SceneImpl &s, const float4 *d_tri, int n, const BuildConfig &cfg,
                    cudaStream_t st);
// Permutes the scene's breadth-first node array (level l = nodes
// [level_start[l], level_start[l + 1])) into depth-first order of child pairs.
int kd_layout_depth_first(SceneImpl &s, const std::vector<int64_t> &level_start, cudaStream_t st);
int sm_count(int device);

}  // namespace xyzgpu
