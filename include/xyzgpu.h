/* xyzgpu: B200 (sm_100a) path-tracing hot path of the xyz renderer behind a C ABI.
 *
 * The reference renderer (goofoo/xyz) exposes its hot path as the C++ singleton
 * `xyz::Scene` driven by an integrator thread:
 *   Scene::Load / Scene::Build                    xyz/core/scene.hpp:51-52
 *   Scene::FindIntersection (closest hit)         xyz/core/scene.hpp:236-238, 277-295
 *   Scene::EvalutePathTracing (one path sample)   xyz/core/scene.hpp:56-58
 *   PathTracer::run (spp x pixel loop, film +=)   xyz/integrator/integrator.cpp:88-162
 * This header is the batch form of those calls.  Every function returns 0 or a
 * negative XYZGPU_E_* code; no exception crosses the ABI; the message of the
 * last failure on the calling thread is xyzgpu_last_error().  The reference has
 * no status codes (it prints to stderr and returns early,
 * xyz/core/scene.cpp:47-51); invalid input here is an error instead.
 *
 * Conventions (same as the reference unless stated):
 *  - Triangles are double-faced; the front normal of (v0, v1, v2) is
 *    normalize(cross(v2 - v0, v1 - v0))  (xyz/geom/triangle.cpp:10-20).
 *  - Materials are Lambert (XYZ albedo) or light.  Lights radiate from their
 *    front side only and share one power Phi (XYZ) spread over the total light
 *    area as radiance Phi / (pi * A)  (xyz/core/scene_pathtracing.cpp:81-112).
 *  - Film: W*H*3 floats, CIE XYZ, row y = 0 at the bottom (film[y*W+x]),
 *    holding the SUM over samples (the reference divides by spp when saving,
 *    xyz/core/imagefilm.cpp:90-105).
 *  - Random numbers: Philox4x32-10 (Salmon et al., SC'11) keyed by the seed;
 *    dimension `dim` of sample `s` of pixel `p` is
 *      u = (Philox(ctr = {p, s, dim / 4, 0}, key = {seed, seed >> 32})[dim % 4] >> 8) * 2^-24.
 *    Dimensions are consumed in the order the reference's estimator reads
 *    IPrimarySample::next() (xyz/bsdf/bsdf.hpp:10-14): 0-1 pixel jitter,
 *    2-3 light sample, (thin lens) 4-5 lens sample, then per vertex an optional
 *    Russian-roulette draw and two BSDF draws.
 */
#ifndef XYZGPU_H_
#define XYZGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XYZGPU_ABI_VERSION 1

#define XYZGPU_OK 0
#define XYZGPU_E_INVALID -1   /* bad argument or scene description */
#define XYZGPU_E_CUDA -2      /* CUDA runtime error (message has the CUDA text) */
#define XYZGPU_E_NOMEM -3     /* device or host allocation failed */
#define XYZGPU_E_LIMIT -4     /* size beyond a documented limit */
#define XYZGPU_E_NODEVICE -5  /* no usable sm_100 device */

typedef struct xyzgpu_scene_s *xyzgpu_scene;

/* Scene description, host memory, copied by xyzgpu_scene_create.
 * Replaces Scene::Load (xyz/core/scene_mqo.cpp:547-777), which fills the same
 * triangle / material / light lists from an MQO file. */
typedef struct {
  const float *positions;       /* 3 * n_vertices */
  const float *normals;         /* 3 * n_vertices shading normals, or NULL (flat) */
  int n_vertices;
  const int32_t *triangles;     /* 3 * n_triangles vertex indices */
  const int32_t *tri_material;  /* n_triangles material ids */
  int n_triangles;
  const float *albedo_xyz;      /* 3 * n_materials (ignored for lights) */
  const int32_t *is_light;      /* n_materials flags */
  int n_materials;
  float light_power_xyz[3];     /* Phi shared by all light triangles */
  /* Spectral data for the spectral film modes (else NULL / unused):
   * 31 albedo bins per material at 400, 410, ..., 700 nm and the light's
   * power spectrum (the reference's basic_spectrum, libhi/hi/image/spectrum.hpp:14). */
  const float *albedo_spd;      /* 31 * n_materials, or NULL */
  float light_power_spd[31];
  /* Kinds of the non-light materials (NULL: all Lambert): XYZGPU_MATERIAL_*.
   * MIRROR is the reference's perfect mirror (xyz/bsdf/mirror.cpp: no
   * next-event estimation, the throughput unchanged, a specular bounce);
   * METAL its glossy Neumann-Neumann BRDF with a Phong-lobe half vector of
   * exponent shininess[m], a Schlick-style Fresnel term with F0 = 0.9 and
   * next-event estimation MIS-weighted against that lobe (xyz/bsdf/metal.cpp
   * built with CONFIG_EXPLICIT_GLOSSY); its albedo multiplies the throughput as
   * Lambert's does.  Scenes with MIRROR or METAL render in the XYZ film mode
   * with xyzgpu_render and batches only (xyzgpu_render_noalloc takes MIRROR
   * but refuses METAL, whose shadow records need a per-path array it does
   * not hold; the guided and importance-driven tracers refuse both). */
  const int32_t *material_kind; /* n_materials, or NULL */
  const float *shininess;       /* n_materials (METAL exponent), or NULL */
} xyzgpu_scene_desc;

#define XYZGPU_MATERIAL_LAMBERT 0
#define XYZGPU_MATERIAL_MIRROR 2
#define XYZGPU_MATERIAL_METAL 3

/* kd-tree construction parameters (the reference: KDTree(max_bucket = 16,
 * max_depth = 16), SAH without traversal / intersection constants,
 * xyz/geom/kdtree.hpp:19-20, kdtree.cpp:261-272). */
typedef struct {
  int leaf_max_tris;      /* make a leaf at or below this many triangles (8) */
  int max_depth;          /* depth limit; 0 = 8 + 1.3 * log2(n_triangles) */
  float cost_traversal;   /* SAH traversal cost (1.0) */
  float cost_intersect;   /* SAH intersection cost (1.5) */
  float empty_bonus;      /* SAH discount for a split with an empty side (0) */
  int bins;               /* SAH bins per axis per node (64, the maximum) */
  int builder;            /* XYZGPU_BUILD_DEVICE (default) or XYZGPU_BUILD_HOST */
  int max_refs_factor;    /* reference budget = factor * n_triangles (6) */
} xyzgpu_build_params;

#define XYZGPU_BUILD_DEVICE 0
#define XYZGPU_BUILD_HOST 1

void xyzgpu_build_params_default(xyzgpu_build_params *bp);

/* Uploads the scene and builds its kd-tree (Scene::Load + Scene::Build,
 * xyz/core/scene.cpp:35).  The device is the current CUDA device. */
int xyzgpu_scene_create(const xyzgpu_scene_desc *desc, const xyzgpu_build_params *bp,
                        xyzgpu_scene *out);

/* Frees the scene's device memory. */
void xyzgpu_scene_destroy(xyzgpu_scene scene);

typedef struct {
  int64_t n_triangles, n_lights, n_nodes, n_leaves, n_empty_leaves, n_leaf_refs;
  int64_t max_depth, device_bytes;
  double build_ms;        /* wall time of the last kd-tree build */
  float light_area;
  float bounds_min[3], bounds_max[3];
} xyzgpu_scene_stats;

int xyzgpu_scene_stats_get(xyzgpu_scene scene, xyzgpu_scene_stats *out);

/* Copies the flattened kd-tree to host memory (for inspection and tests).
 * nodes: 2 * n_nodes uint32 (see the node layout in csrc/kdtree.h); refs:
 * n_leaf_refs int32.  Either pointer may be NULL. */
int xyzgpu_scene_copy_tree(xyzgpu_scene scene, uint32_t *nodes, int32_t *refs);

/* Closest hit for a batch of rays: the batch form of Scene::FindIntersection
 * (xyz/core/scene.hpp:277-295 -> KDTree::FindIntersection, kdtree.cpp:366-372;
 * triangle test FindIntersectionDF, triangle.cpp:127-165).
 *   rays: device, n * 8 floats per ray: ox oy oz tmin dx dy dz tmax
 *         (the reference's interval is tmin = 1e-5, tmax = +inf,
 *          xyz/geom/intersection.hpp:11-14)
 *   hits: device, n * 4 words: t, f, g (floats) and an int32
 *         (triangle_id << 1 | back_side), or -1 for a miss.
 *   stream: cudaStream_t or NULL. */
int xyzgpu_trace_closest(xyzgpu_scene scene, const float *rays, int n, float *hits,
                         void *stream);

/* Counters of the instrumented traversal (per batch, summed over rays). */
typedef struct {
  uint64_t rays, nodes_visited, leaves_visited, tri_tests, hits;
} xyzgpu_trace_counters;

/* Same as xyzgpu_trace_closest plus work counters (slower; for roofline
 * accounting outside timed regions).  Synchronises `stream`. */
int xyzgpu_trace_closest_counted(xyzgpu_scene scene, const float *rays, int n, float *hits,
                                 void *stream, xyzgpu_trace_counters *counters);

/* Camera as the reference models it (xyz/core/thinlenscamera.cpp:20-28, 71-90):
 * eye, gaze point, film size, focal length, F-number; up = +y.  pinhole != 0
 * selects the CONFIG_PINHOLE_CAMERA_MODEL ray generation (thinlenscamera.cpp:
 * 111-124), otherwise the thin lens (:159-205). */
typedef struct {
  float eye[3];
  float at[3];
  float film_size;
  float focal_length;
  float f_number;
  int pinhole;
} xyzgpu_camera;

#define XYZGPU_FILM_DEVICE 0
#define XYZGPU_FILM_HOST 1

typedef struct {
  int width, height;
  int spp;                 /* samples per pixel rendered by this call */
  int spp_offset;          /* index of the first sample (progressive rendering) */
  int max_depth;           /* max path segments; the reference's kMax - 1 (15) */
  int rr_start_depth;      /* first vertex that plays Russian roulette (1) */
  float rr_threshold;      /* Russian roulette on throughput Y below this (0.2) */
  uint64_t seed;
  int film_location;       /* XYZGPU_FILM_DEVICE or XYZGPU_FILM_HOST */
  int accumulate;          /* nonzero: add into film; zero: overwrite */
  int wave_paths;          /* paths in flight per wave; 0 = every path of the call,
                              at most 2^26, bounded by half of the free device memory.
                              Wave buffers are shared by all scenes of a device. */
  int profile;             /* XYZGPU_PROFILE_*: per-kernel timing or work counters */
  int spectral;            /* XYZGPU_SPECTRAL_*: XYZ tristimulus paths (the xyz renderer,
                              default) or hero-wavelength spectral paths */
  int hero_wavelengths;    /* 1..4 wavelengths per path in the spectral modes */
  int row_begin, row_end;  /* render only image rows [row_begin, row_end) (a band of the same
                              image: same pixels, same paths); 0, 0 = all rows */
  int row_step;            /* with a band: render only rows row_begin + k * row_step (0 or 1:
                              every row of the band); rows not rendered hold zero (or keep
                              their values when accumulating), as outside a band */
} xyzgpu_render_params;

/* Film modes.  OFF: throughput and albedo are CIE XYZ triples, the estimator of
 * xyz::Scene::EvalutePathTracing.  BINNED: the estimator of the reference's
 * spectral renderer, tgir::Scene::EvaluteRussianRoulette
 * (renderer/core/SceneStrategy.cpp:11-149): one of 31 equal-probability bins
 * over 400..700 nm per wavelength, next-event estimation before the depth cap,
 * Russian roulette on the first wavelength's throughput, XYZ = L * 31 * CMF[bin]
 * (libhi/hi/image/spectrum.cpp:561-567); hero_wavelengths = 1 is that
 * estimator exactly.  CONTINUOUS: the same estimator with wavelengths uniform in
 * 380..720 nm and spectra interpolated as basic_spectrum::Sample does
 * (spectrum.cpp:148-165, clamped to the end bins outside 400..700).  Hero
 * wavelength j of a path is frac(u + j / H), u the path's wavelength draw
 * (the dimension after the camera's). */
#define XYZGPU_SPECTRAL_OFF 0
#define XYZGPU_SPECTRAL_BINNED 1
#define XYZGPU_SPECTRAL_CONTINUOUS 2

#define XYZGPU_PROFILE_OFF 0
#define XYZGPU_PROFILE_TIMING 1   /* CUDA events around every kernel launch */
#define XYZGPU_PROFILE_COUNTERS 2 /* traversal work counters (slower kernels) */

void xyzgpu_render_params_default(xyzgpu_render_params *rp);

/* Renders rp->spp samples per pixel (PathTracer::run's loop around
 * Scene::EvalutePathTracing, xyz/integrator/integrator.cpp:119-128) into
 * `film` (W*H*3 XYZ sums).  Wavefront: ray generation, closest hit, shading
 * (emitter MIS, next-event estimation, Russian roulette, Lambert sampling),
 * shadow rays and film accumulation are separate kernels over SoA queues.
 * A host film is copied in and out inside the call: directly when it is in
 * page-locked memory (cudaMallocHost, cudaHostRegister), else through a pinned
 * staging buffer. */
int xyzgpu_render(xyzgpu_scene scene, const xyzgpu_camera *camera,
                  const xyzgpu_render_params *rp, float *film, void *stream);

typedef struct {
  uint64_t paths, extension_rays, shadow_rays, shadow_hits_visible, waves, kernel_launches;
} xyzgpu_render_counters;

/* Counters of the last xyzgpu_render on this scene (synchronises). */
int xyzgpu_render_counters_get(xyzgpu_scene scene, xyzgpu_render_counters *out);

/* Per-kernel-class profile of the last xyzgpu_render (or
 * xyzgpu_render_guided) that had profile != 0 (synchronises).  Classes:
 * 0 raygen, 1 extension trace, 2 shade, 3 shadow trace, 4 film, 5 guide
 * (network inference per bounce and, in training renders, the training
 * records and Adam steps).  ms: summed CUDA-event time (TIMING); the
 * traversal counters are filled by a COUNTERS render. */
#define XYZGPU_KERNEL_CLASSES 6
#define XYZGPU_PROFILE_MAX_ITERS 64
typedef struct {
  uint64_t launches[XYZGPU_KERNEL_CLASSES];
  double ms[XYZGPU_KERNEL_CLASSES];
  uint64_t ext_rays, ext_nodes, ext_leaves, ext_tri_tests;
  uint64_t shadow_rays, shadow_nodes, shadow_leaves, shadow_tri_tests, shadow_visible;
  uint32_t iterations;          /* bounce iterations per wave (max_depth) */
  uint64_t ext_rays_by_iter[XYZGPU_PROFILE_MAX_ITERS];     /* summed over waves */
  uint64_t shadow_rays_by_iter[XYZGPU_PROFILE_MAX_ITERS];
} xyzgpu_render_profile;

int xyzgpu_render_profile_get(xyzgpu_scene scene, xyzgpu_render_profile *out);

/* Rendering without allocation.  No counterpart in the reference (which
 * renders on the CPU and never allocates GPU memory); it exists for callers
 * that cannot allocate device memory while running - an application that
 * gives all GPU memory to its own pool at start-up, a real-time loop that may
 * not call the allocator mid-frame, a process with a fixed memory budget.
 * Same image as xyzgpu_render for the same parameters, but the path state and
 * queues live in one file-scope device array of XYZGPU_NOALLOC_SCRATCH_BYTES
 * that every device loading the library holds until exit, so at most
 * XYZGPU_NOALLOC_MAX_WAVE_PATHS paths are in flight at a time.
 * Limits (else XYZGPU_E_LIMIT / XYZGPU_E_INVALID): film in device memory,
 * max_depth <= XYZGPU_NOALLOC_MAX_DEPTH, wave_paths <= the wave maximum,
 * profile off.  The first call on a device looks up the array's address
 * (make that first call before any stream capture).  All calls share the
 * array: calls that overlap on the GPU race and must be serialised.
 * Allocates nothing: no cudaMalloc, cudaFree or host allocation of pinned
 * memory. */
#define XYZGPU_NOALLOC_MAX_WAVE_PATHS 65536
#define XYZGPU_NOALLOC_MAX_DEPTH 64
#define XYZGPU_NOALLOC_SCRATCH_BYTES 11536896
/* (XYZ film mode only.) */
int xyzgpu_render_noalloc(xyzgpu_scene scene, const xyzgpu_camera *camera,
                          const xyzgpu_render_params *rp, float *film_device, void *stream);

/* Material parameters after creation (the differentiable-rendering inputs).
 * albedo_xyz: 3 per material (the XYZ triple the throughput is multiplied by;
 * ignored for lights); emission: 1 per material, a scale of the light power
 * emitted by that material's light triangles (1 at creation, so the emitted
 * radiance is the reference's Phi / (pi * light area) until it is set; an
 * extension: the reference has one power for all lights).  Either pointer may
 * be NULL (left unchanged).  location: XYZGPU_FILM_HOST (values checked and
 * copied before return) or XYZGPU_FILM_DEVICE (device arrays read on
 * `stream`, not checked). */
int xyzgpu_scene_set_materials(xyzgpu_scene scene, const float *albedo_xyz, const float *emission,
                               int location, void *stream);

/* Copies the current material parameters to host arrays (either may be NULL). */
int xyzgpu_scene_get_materials(xyzgpu_scene scene, float *albedo_xyz, float *emission);

/* Path-replay adjoint of xyzgpu_render (Vicini, Speierer and Jakob, "Path
 * Replay Backpropagation", 2021).  With film = the W*H*3 sums xyzgpu_render
 * produces for the same scene, camera and parameters, adds
 *   d_albedo[3m + c] += sum_p d_film[p] . d film[p] / d albedo[m][c]
 *   d_emission[m]    += sum_p d_film[p] . d film[p] / d emission[m]
 * for the same sample paths (same seed and sample indices): each wave runs
 * twice, a primal pass that keeps every path's radiance and a replay pass that
 * regenerates the same paths and, at each vertex, scatters
 * d_film . (radiance collected from that vertex on) / albedo into the vertex's
 * material and d_film . (emitted contribution at unit scale) into the light's.
 * The primal pass also records each path's closest hit and shadow-ray result
 * per bounce (20 bytes per path and bounce, stream-ordered device memory), and
 * the replay reads them instead of tracing rays; when that memory cannot be
 * had, or the environment variable XYZGPU_ADJOINT_TRACE_REPLAY is set, the
 * replay traces its paths again (same result).
 * The path sampling (Lambert cosine lobe, light choice by area, MIS weights) does
 * not depend on albedo or emission, so with Russian roulette off
 * (rr_threshold = 0) the result is the exact derivative of the rendered film;
 * with it on, the roulette's survival scale is held constant.  An albedo channel
 * that is exactly 0 gets no gradient from vertices of that material.
 * d_film, d_albedo (3 * n_materials) and d_emission (n_materials) are device
 * arrays; gradients are accumulated with float atomics (summation order varies
 * between calls).  XYZ film mode only, profile off; film_location and
 * accumulate are ignored. */
int xyzgpu_adjoint(xyzgpu_scene scene, const xyzgpu_camera *camera,
                   const xyzgpu_render_params *rp, const float *d_film, float *d_albedo,
                   float *d_emission, void *stream);

/* Batched rendering: many scenes of different size, resolution and sample count
 * rendered together.  No counterpart in the reference, which renders one scene
 * per process.  Every kernel launch serves all jobs at once: one wave of paths
 * holds runs of consecutive samples of several jobs ("blocks"), and each path
 * carries its block, so traversal, shading and film kernels fetch the scene,
 * camera and estimator parameters per path.  A job renders the same film as
 * xyzgpu_render with its parameters (same paths, same per-pixel sample order).
 * xyzgpu_batch_launch is one cudaGraphLaunch of a graph captured at creation
 * whose loops over the waves and over each wave's bounces are conditional
 * (WHILE) nodes run by the device: the kernels read the current wave and
 * bounce from device memory, so the graph has the same few nodes however many
 * waves the batch has, and a wave's bounce loop ends when its rays run out. */
typedef struct {
  xyzgpu_scene scene;            /* must outlive the batch */
  xyzgpu_camera camera;
  xyzgpu_render_params params;   /* XYZ film mode, profile off; film_location and
                                    wave_paths are ignored (the film is device memory) */
  float *film;                   /* device, width * height * 3 sums */
} xyzgpu_batch_job;

typedef struct {
  int wave_paths;          /* paths in flight per wave (the queue capacity); 0 = default
                              (all paths, at most 2^24); at least the largest job's
                              pixel count */
  int tile;                /* slot order of a job's pixels: tiles of tile x tile pixels
                              (1 = scanlines); jobs whose size is not a multiple use 1 */
  int trace_ctas_per_sm;   /* CTAs per SM of the persistent trace kernels; 0 = the
                              occupancy maximum */
  int use_graph;           /* nonzero: replay a captured CUDA graph (default 1) */
} xyzgpu_batch_config;

typedef struct xyzgpu_batch_s *xyzgpu_batch;

void xyzgpu_batch_config_default(xyzgpu_batch_config *cfg);

/* Plans the waves, allocates the batch's own path buffers and, with use_graph,
 * captures the launch sequence.  cfg may be NULL (defaults). */
int xyzgpu_batch_create(const xyzgpu_batch_job *jobs, int n_jobs, const xyzgpu_batch_config *cfg,
                        xyzgpu_batch *out);

/* Renders every job's spp samples into its film (film zeroed first unless the
 * job's accumulate is set).  Asynchronous on `stream`. */
int xyzgpu_batch_launch(xyzgpu_batch batch, void *stream);

/* Sets each job's first sample index (progressive rendering: launch, then move
 * the offsets by spp, launch again).  Takes effect at the next launch. */
int xyzgpu_batch_set_sample_offsets(xyzgpu_batch batch, const uint32_t *spp_offsets);

/* Autotuner: times launches of candidate configurations on this batch (tile,
 * wave size, trace CTAs per SM; coordinate descent from the current one, each
 * candidate timed `trials` times with CUDA events, best kept) and re-plans with
 * the winner.  probe_spp > 0 caps every job's samples during the search.  The
 * films are not touched (scratch films).  Synchronises `stream`. */
int xyzgpu_batch_autotune(xyzgpu_batch batch, int trials, int probe_spp, void *stream,
                          xyzgpu_batch_config *chosen);

typedef struct {
  uint64_t paths, waves, kernel_launches_per_launch, extension_rays, shadow_rays;
  int64_t device_bytes;     /* path buffers, tables and scratch of the batch */
  int graph_nodes;          /* nodes of the captured graph, its loop bodies included
                               (0 without a graph) */
  int graph_top_nodes;      /* nodes at the graph's top level: the start kernel and
                               the wave loop */
} xyzgpu_batch_stats;

/* Statistics of the batch; ray and kernel counts are those of the last launch
 * (synchronises). */
int xyzgpu_batch_stats_get(xyzgpu_batch batch, xyzgpu_batch_stats *out);

int xyzgpu_batch_config_get(xyzgpu_batch batch, xyzgpu_batch_config *out);

void xyzgpu_batch_destroy(xyzgpu_batch batch);

/* One-shot form: create, launch, synchronise, destroy. */
int xyzgpu_render_batch(const xyzgpu_batch_job *jobs, int n_jobs, const xyzgpu_batch_config *cfg,
                        void *stream);

/* Learned path guide: an MLP from a surface point (position, normal) to an
 * 8-lobe von Mises-Fisher mixture over directions, trained online on the
 * tracer's own radiance samples and combined with Lambert sampling by one-
 * sample MIS (so the estimator stays unbiased).  No counterpart in the
 * reference; its non-learned analogue is the importon histogram of
 * xyz/core/photonmap.cpp:365-494.  The network: one-blob encoding (32 bins per
 * input, 192 values), four hidden layers of 64 with ReLU, 64 outputs (0..7
 * mixture logits, 8..15 log concentrations clamped to [-5, 8], 16..39 lobe
 * means, 40..63 unused); bf16 weights, fp32 accumulation on tcgen05 tensor
 * cores; Adam on fp32 master weights.  Parameters (XYZGPU_GUIDE_PARAMS floats):
 * for each layer l = 0..4, W_l as [in][64] row-major then b_l[64]. */
#define XYZGPU_GUIDE_PARAMS 28992
#define XYZGPU_GUIDE_OUTPUTS 64

typedef struct {
  float alpha;           /* probability of sampling the guide in the one-sample MIS (0.5) */
  float learning_rate;   /* Adam step size (1e-3) */
  int batch_size;        /* training records per Adam step (65536) */
  int steps_per_pass;    /* Adam steps after each training render (16) */
  int train_bounces;     /* path vertices per path that give training records (2) */
  uint64_t seed;         /* weight initialisation */
  int guide_bounces;     /* path vertices sampled with the guide (the first ones); deeper
                            vertices use Lambert sampling alone and need no inference (4) */
} xyzgpu_guide_config;

typedef struct xyzgpu_guide_s *xyzgpu_guide;

void xyzgpu_guide_config_default(xyzgpu_guide_config *cfg);
/* A guide for `scene` (positions are normalised by its bounds). */
int xyzgpu_guide_create(xyzgpu_scene scene, const xyzgpu_guide_config *cfg, xyzgpu_guide *out);
void xyzgpu_guide_destroy(xyzgpu_guide guide);
/* fp32 master parameters, host arrays of XYZGPU_GUIDE_PARAMS (set resets Adam). */
int xyzgpu_guide_get_params(xyzgpu_guide guide, float *params);
int xyzgpu_guide_set_params(xyzgpu_guide guide, const float *params);
/* Network outputs for n points: features n x 6 (position, normal), out n x 64
 * (device arrays).  Synchronises `stream`. */
int xyzgpu_guide_forward(xyzgpu_guide guide, const float *features, int n, float *out, void *stream);
/* Adds scale * d/dparams sum_i -w_i log p(d_i | x_i) to grad (device,
 * XYZGPU_GUIDE_PARAMS floats); records: n x 10 = position, normal, direction
 * d (unit), weight w (device).  Synchronises `stream`. */
int xyzgpu_guide_gradient(xyzgpu_guide guide, const float *records, int n, float scale, float *grad,
                          void *stream);
/* One Adam step on the mean loss of n records.  Synchronises `stream`. */
int xyzgpu_guide_train_step(xyzgpu_guide guide, const float *records, int n, void *stream);

/* Guided render: as xyzgpu_render (XYZ film mode) with every Lambert vertex
 * sampled from the one-sample MIS of the guide (probability alpha) and the
 * cosine lobe, and the next-event MIS weights computed with that mixture
 * density, so the estimator stays unbiased whatever the network outputs.  Per
 * bounce the wavefront runs closest hit, guide inference on the tensor cores
 * (a mixture per queue entry), shading and shadow rays.  train != 0: the first
 * train_bounces vertices of every path also leave training records (point,
 * sampled direction, incident-radiance weight), and after each wave the guide
 * takes steps_per_pass Adam steps on them.  Russian
 * roulette tests the throughput the path would have with Lambert sampling (the
 * throughput times the product of the guide / Lambert density ratios): the
 * guide sends paths towards bright regions with a high pdf, i.e. a low
 * throughput, which roulette on the throughput itself would end.  A training
 * wave's records, Adam steps and bookkeeping run on the device as one CUDA
 * graph (captured on a private stream the first time a wave of that size
 * trains), so training enqueues no host synchronisation. */
int xyzgpu_render_guided(xyzgpu_guide guide, const xyzgpu_camera *camera,
                         const xyzgpu_render_params *rp, int train, float *film, void *stream);

/* Allocates the guided-wave buffers now - the mixtures (80 B per path) and,
 * with train, the training records and rows (520 B per path at 5 training
 * bounces) - for waves of up to wave_paths paths (at most 2^23, the guided
 * wave size), so that xyzgpu_render_guided calls whose waves fit allocate
 * nothing (else the first such call allocates them).  No counterpart in the
 * reference.  Synchronises `stream`. */
int xyzgpu_guide_reserve(xyzgpu_guide guide, int64_t wave_paths, int train, void *stream);

typedef struct {
  uint64_t adam_steps, trained_records;
} xyzgpu_guide_stats;

int xyzgpu_guide_stats_get(xyzgpu_guide guide, xyzgpu_guide_stats *out);

/* ---- Importance-driven path tracing: the reference's non-learned path guide,
 * Scene::EvaluteImportanceDrivenPathTracing (xyz/core/
 * scene_importancedrivenpathtracing.cpp:11-180).  Light particles are traced
 * first and leave "importons" (hit point, incoming direction) on Lambert
 * surfaces (Scene::CreateLightImportanceMap, xyz/core/scene_photonmap.cpp:
 * 272-330); at a path vertex the importons within `radius` give a 16-bin
 * histogram over (cos^2 theta, phi) about the shading frame, every bin
 * starting at 16 counts (ImportanceQuery, xyz/core/photonmap.cpp:321-439);
 * the next direction is drawn from it (the throughput divided by the bin's
 * density) and next-event estimation's MIS weight uses its density.  As the
 * variants that act in Lambert-only scenes: importons at every Lambert hit
 * from bounce min_depth on (the source keeps only those after a specular
 * bounce), histogram sampling at every Lambert vertex of the first
 * guide_bounces (the source's "[TEST]" condition; it uses it only after a
 * specular bounce).  Particle p reads the Philox stream (pixel = p,
 * sample = 0xffffffff): two draws for the light point, two for a cosine
 * direction about the light's geometric normal, then per Lambert hit a
 * roulette draw (survival albedo.y, Lambert::BoundsImportance) and two for the
 * next cosine direction about the geometric normal.  At a guided vertex the
 * path reads one draw for the bin and two inside it (after the optional
 * roulette draw) instead of the two of cosine sampling. */
typedef struct {
  int particles;       /* light particles (100,000: CONFIG_EMITED_SIZE, xyz/core/config.hpp:57) */
  int max_depth;       /* bounces per particle (16: the reference's kMax) */
  int min_depth;       /* keep importons from this bounce on (1) */
  float radius;        /* search radius (0.1: CONFIG_SEARCH_RADIUS, config.hpp:56) */
  uint64_t seed;
  int guide_bounces;   /* path vertices sampled from the histogram (the first ones); deeper
                          vertices use cosine sampling (default: all) */
} xyzgpu_importon_config;

typedef struct xyzgpu_importons_s *xyzgpu_importons;

void xyzgpu_importon_config_default(xyzgpu_importon_config *cfg);
/* Builds the map of `scene`: traces cfg->particles light particles, or - with
 * importons != NULL - takes the n_importons given ones (6 floats each:
 * position, incoming direction; host memory).  Synchronises `stream`. */
int xyzgpu_importons_create(xyzgpu_scene scene, const xyzgpu_importon_config *cfg, const float *importons,
                            int64_t n_importons, void *stream, xyzgpu_importons *out);
void xyzgpu_importons_destroy(xyzgpu_importons map);
/* Number of importons, and with importons != NULL a host copy (6 floats each,
 * in the map's cell order). */
int xyzgpu_importons_get(xyzgpu_importons map, float *importons, int64_t *n);
/* Histograms for n frames (device, 12 floats each: position, tangent,
 * binormal, shading normal): hist (device) gets 16 cumulative bin counts per
 * frame, bins u * 8 + v for u = floor(2 cos^2 theta), v = floor(8 phi / 2 pi). */
int xyzgpu_importons_query(xyzgpu_importons map, const float *frames, int n, float *hist, void *stream);
/* As xyzgpu_render (XYZ film mode; profile off or timing, class 5 = the
 * histogram queries) with the importance-driven estimator. */
int xyzgpu_render_importon(xyzgpu_importons map, const xyzgpu_camera *camera, const xyzgpu_render_params *rp,
                           float *film, void *stream);

/* ---- Film output.  Post-processing on the device of a film as xyzgpu_render
 * leaves it (W * H XYZ sums, row 0 at the bottom, device memory), and the
 * files around it. */

/* Radiance RGBE pixels of ImageFilm::SaveAsHdr (xyz/core/imagefilm_hdr.cpp:
 * 124-183): pixel = film * scale (scale = 1 / spp), converted to CCIR 601-1 RGB
 * (a non-finite pixel becomes 0) and encoded as hdr_encode does (:14-31);
 * out: W * H * 4 bytes (device) in file order, scanlines from the top image
 * row down.  xyze != 0: the reference's CONFIG_HDR_STRICT output, XYZ encoded
 * directly, scanlines from the bottom row up. */
int xyzgpu_film_encode_rgbe(const float *film, int width, int height, float scale, int xyze, uint8_t *out,
                            void *stream);

/* Writes a Radiance .hdr file (header and run-length scanlines, the format of
 * imagefilm_hdr.cpp:46-183) from the host copy of xyzgpu_film_encode_rgbe's
 * output. */
int xyzgpu_hdr_write(const char *path, const uint8_t *rgbe, int width, int height, int xyze);

/* Tone operators of the reference's float2bmp tool (float2bmp/main.cpp:80-118)
 * applied per channel: FILM 1 - exp(-exposure L) (the one the tool uses),
 * LINEAR exposure L, REINHARD exposure L / (1 + L), REINHARD_WHITE
 * exposure L (1 + L / white^2) / (1 + L); then L^(src_gamma / dst_gamma) and
 * the 8-bit quantisation min(255, floor(256 v)) for v in (0, 1). */
#define XYZGPU_TONEMAP_FILM 0
#define XYZGPU_TONEMAP_LINEAR 1
#define XYZGPU_TONEMAP_REINHARD 2
#define XYZGPU_TONEMAP_REINHARD_WHITE 3
typedef struct {
  float scale;       /* film multiplier (1 / spp) */
  int op;            /* XYZGPU_TONEMAP_* */
  float exposure;    /* (1, the tool's default) */
  float white;       /* REINHARD_WHITE: white point; <= 0: the image's maximum of
                        0.6069 c0 + 0.1735 c1 + 0.2003 c2, as the tool computes it */
  float dst_gamma;   /* 2.2 */
  float src_gamma;   /* 1.0 */
  int rgb;           /* 0: the film's channels as they are (the tool reads the
                        reference's .pfm, which holds XYZ); 1: CCIR 601-1 RGB */
} xyzgpu_tonemap_params;

void xyzgpu_tonemap_params_default(xyzgpu_tonemap_params *tp);

/* 24-bit BMP pixel rows (device): rows from the bottom, bytes blue, green, red
 * = tone-mapped channels 2, 1, 0 (the tool's order), each row padded to a
 * multiple of 4 bytes.  scratch_white: one device word, needed only for
 * REINHARD_WHITE with white <= 0. */
int xyzgpu_film_tonemap(const float *film, int width, int height, const xyzgpu_tonemap_params *tp, uint8_t *out,
                        unsigned int *scratch_white, void *stream);

/* Writes a 24-bit BMP file (the header of float2bmp/main.cpp:131-144) from the
 * host copy of xyzgpu_film_tonemap's output. */
int xyzgpu_bmp_write(const char *path, const uint8_t *bgr, int width, int height);

/* Host-film forms: the film (host, W * H * 3 sums) is uploaded, encoded or
 * tone-mapped by the kernels above and written (synchronous; allocates device
 * memory for the call).  save_hdr is the reference's ImageFilm::SaveAsHdr with
 * mpp = spp; save_bmp is float2bmp applied to the film. */
int xyzgpu_film_save_hdr(const char *path, const float *film, int width, int height, float spp, int xyze);
int xyzgpu_film_save_bmp(const char *path, const float *film, int width, int height,
                         const xyzgpu_tonemap_params *tp);

/* Resumable render checkpoint (no counterpart in the reference, whose periodic
 * .pfm dump, xyz/integrator/integrator.cpp:140-160, keeps the image but not
 * the means to continue it): the film sums (host memory, W * H * 3 floats),
 * the number of samples per pixel done and the render parameters, with a
 * checksum of the film.  To resume, load, then render with
 * spp_offset = spp_done and accumulate = 1 into the loaded film: the film
 * kernels add each path's sample into the pixel in sample order, so the
 * resumed film is bit-identical to an uninterrupted render.  The file is
 * written under a temporary name and renamed, so a crash never leaves a
 * half-written checkpoint.  load with film = NULL reads only the header. */
int xyzgpu_checkpoint_save(const char *path, const xyzgpu_render_params *rp, int spp_done, const float *film);
int xyzgpu_checkpoint_load(const char *path, xyzgpu_render_params *rp, int *spp_done, float *film);

/* ---- Spectral tables on the host (for scene loaders and tools).  The named
 * spectra of the reference's library (libhi/hi/image/spectrum.cpp:170-476),
 * 31 bins at 400, 410, ..., 700 nm: illuminants "light_source_a",
 * "light_source_b", "light_source_c", "light_d65", "light_d100",
 * "light_standard_warm_white", "light_white", "light_standard_white",
 * "light_daylight", "light_warm_white_de_luxe", "light_soft_white",
 * "light_cool_white_de_luxe", "light_mercury_arc_lamp" and the 24 Macbeth
 * ColorChecker patches "mcc_dark_skin" ... "mcc_black" (reflectances).
 * Returns XYZGPU_E_INVALID for an unknown name. */
int xyzgpu_named_spectrum(const char *name, float out[31]);
/* hi::spd2xyz (spectrum.cpp:554-559): the spectrum's XYZ through the CIE 1931
 * colour-matching functions (float dot products in bin order). */
void xyzgpu_spectrum_to_xyz(const float spd[31], float xyz[3]);

/* Host evaluation of the random stream defined above (for tests). */
float xyzgpu_philox_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t dim);

const char *xyzgpu_last_error(void);
int xyzgpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* XYZGPU_H_ */
