// C ABI of the path-tracing library (declarations and reference citations in
// include/xyzgpu.h): argument checking, scene upload and kd-tree build
// dispatch, error reporting.  Kernels live in trace.cu, render.cu, kdbuild.cu.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "scene.h"

namespace xyzgpu {

namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

int sm_count(int device) {
  static int cached[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (cached[device] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
      v = 148;
    cached[device] = v;
  }
  return cached[device];
}

namespace {

// Scene and builder memory comes from the device's stream-ordered pool, which
// keeps freed blocks for reuse: building and destroying scenes repeatedly
// (batches, end-to-end loops) then costs no driver allocation or device-wide
// synchronisation after the first time.
void configure_pool(int device) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~uint64_t{0};
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done[device] = true;
}

template <class T>
int dev_alloc(T **dst, size_t n, int64_t *bytes, cudaStream_t st) {
  n = n ? n : 1;
  XYZ_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(dst), n * sizeof(T), st));
  *bytes += static_cast<int64_t>(n * sizeof(T));
  return XYZGPU_OK;
}

template <class T>
int dev_upload(T **dst, const T *src, size_t n, int64_t *bytes, cudaStream_t st) {
  int const rc = dev_alloc(dst, n, bytes, st);
  if (rc) return rc;
  if (n) XYZ_CUDA_TRY(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
  return XYZGPU_OK;
}

void free_scene(SceneImpl *s) {
  if (!s) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  // work queued on any stream that still reads the scene finishes first
  cudaDeviceSynchronize();
  render_workspace_free(s->ws);
  void *bufs[] = {s->d_tri, s->d_ng, s->d_sn, s->d_mat, s->d_shininess, s->d_emission, s->d_lights, s->d_cdf, s->d_spd,
                  s->d_nodes, s->d_refs, s->d_fetch, s->d_trace_counts};
  for (void *b : bufs)
    if (b) cudaFreeAsync(b, nullptr);
  cudaStreamSynchronize(nullptr);
  cudaSetDevice(prev);
  delete s;
}

// Triangle records from the uploaded vertex and index arrays (the Triangle
// constructor, xyz/geom/triangle.cpp:35-60): v0, e1 = v1 - v0, e2 = v2 - v0,
// n = cross(e2, e1), ng = n / |n|, shading normals n0, s1 = n1 - n0,
// s2 = n2 - n0.  Same float operations as the host (--fmad=false).
// Vertex or material indices out of range set flag bit 2 and leave the
// triangle out (nothing is read through them); light_flag[i] marks the
// triangles of light materials.
__global__ void k_prepare_triangles(const float *__restrict__ pos, const float *__restrict__ nrm,
                                    const int32_t *__restrict__ idx, const int32_t *__restrict__ tmat,
                                    int nt, int nv, int nm, const int32_t *__restrict__ is_light,
                                    float4 *__restrict__ tri, float4 *__restrict__ ng,
                                    float4 *__restrict__ sn, float *__restrict__ box_min,
                                    float *__restrict__ box_max, int *flag, int8_t *__restrict__ light_flag) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool valid = false;
  if (i < nt) {
    int const a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
    int const m = tmat[i];
    valid = a >= 0 && b >= 0 && c >= 0 && a < nv && b < nv && c < nv && m >= 0 && m < nm;
    light_flag[i] = valid && is_light[m] != 0;
    if (!valid) atomicOr(flag, 2);
  }
  if (valid) {
    int const a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
    f3 const p0 = mk3(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]);
    f3 const p1 = mk3(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
    f3 const p2 = mk3(pos[3 * c], pos[3 * c + 1], pos[3 * c + 2]);
    f3 const e1 = sub3(p1, p0), e2 = sub3(p2, p0);
    f3 const n = cross3(e2, e1);
    float const r = 1.0f / sqrtf(dot3(n, n));
    tri[3 * i + 0] = make_float4(p0.x, p0.y, p0.z, n.x);
    tri[3 * i + 1] = make_float4(e1.x, e1.y, e1.z, n.y);
    tri[3 * i + 2] = make_float4(e2.x, e2.y, e2.z, n.z);
    ng[i] = make_float4(n.x * r, n.y * r, n.z * r, __int_as_float(tmat[i]));
    if (sn) {
      f3 const n0 = mk3(nrm[3 * a], nrm[3 * a + 1], nrm[3 * a + 2]);
      f3 const n1 = mk3(nrm[3 * b], nrm[3 * b + 1], nrm[3 * b + 2]);
      f3 const n2 = mk3(nrm[3 * c], nrm[3 * c + 1], nrm[3 * c + 2]);
      f3 const s1 = sub3(n1, n0), s2 = sub3(n2, n0);
      sn[3 * i + 0] = make_float4(n0.x, n0.y, n0.z, 0.0f);
      sn[3 * i + 1] = make_float4(s1.x, s1.y, s1.z, 0.0f);
      sn[3 * i + 2] = make_float4(s2.x, s2.y, s2.z, 0.0f);
    }
    // the vertices as the intersection test sees them: v0, v0 + e1, v0 + e2
    f3 const q1 = add3(p0, e1), q2 = add3(p0, e2);
    float const v[3][3] = {{p0.x, p0.y, p0.z}, {q1.x, q1.y, q1.z}, {q2.x, q2.y, q2.z}};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fminf(fminf(v[0][k], v[1][k]), v[2][k]);
      hi[k] = fmaxf(fmaxf(v[0][k], v[1][k]), v[2][k]);
    }
  }
  // scene bounds: block reduction, then one ordered-integer atomic per block
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float l = lo[k], h = hi[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      l = fminf(l, __shfl_xor_sync(0xffffffffu, l, off));
      h = fmaxf(h, __shfl_xor_sync(0xffffffffu, h, off));
    }
    if ((threadIdx.x & 31) == 0 && l <= h) {
      // IEEE order = signed-integer order for non-negative floats, reversed for negative
      int const li = __float_as_int(l), hv = __float_as_int(h);
      if (li >= 0)
        atomicMin(reinterpret_cast<int *>(&box_min[k]), li);
      else
        atomicMax(reinterpret_cast<unsigned *>(&box_min[k]), static_cast<unsigned>(li));
      if (hv >= 0)
        atomicMax(reinterpret_cast<int *>(&box_max[k]), hv);
      else
        atomicMin(reinterpret_cast<unsigned *>(&box_max[k]), static_cast<unsigned>(hv));
    }
  }
}

// Finite coordinates (flag bit 1).
__global__ void k_check_finite(const float *__restrict__ p, int64_t n, int *flag) {
  bool bad = false;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    bad = bad || !isfinite(p[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// The caller's geometry checked on the host, for the message of the first
// fault (run only when the device checks found one): the same order and
// wording as the checks the device made.
int host_geometry_error(const xyzgpu_scene_desc *d) {
  int const nt = d->n_triangles, nv = d->n_vertices, nm = d->n_materials;
  for (int64_t i = 0; i < 3ll * nv; ++i)
    if (!std::isfinite(d->positions[i]))
      return set_error(XYZGPU_E_INVALID, "scene_create: vertex coordinate %lld is not finite",
                       static_cast<long long>(i));
  for (int i = 0; i < nt; ++i) {
    int32_t const a = d->triangles[3 * i], b = d->triangles[3 * i + 1], c = d->triangles[3 * i + 2];
    int32_t const m = d->tri_material[i];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv)
      return set_error(XYZGPU_E_INVALID, "scene_create: triangle %d has a vertex index out of range", i);
    if (m < 0 || m >= nm)
      return set_error(XYZGPU_E_INVALID, "scene_create: triangle %d has material %d out of range", i, m);
  }
  return set_error(XYZGPU_E_INVALID, "scene_create: invalid geometry");
}

int check_device(int *dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return set_error(XYZGPU_E_NODEVICE, "no CUDA device: %s",
                     e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
  XYZ_CUDA_TRY(cudaGetDevice(dev));
  int major = 0;
  XYZ_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, *dev));
  if (major != 10)
    return set_error(XYZGPU_E_NODEVICE, "device %d has compute capability %d.x; this library is built for sm_100a",
                     *dev, major);
  return XYZGPU_OK;
}

// Material table update from device arrays: albedo (3 per material) into the
// xyz of the float4 records, emission scale copied as is.
// The material table from the caller's arrays (uploaded as they are): per
// material (albedo XYZ, w) with w = 1 for a light, the kind for a mirror or
// metal, else 0; the metal exponent (1 elsewhere); emission scale 1.  n = 0
// leaves one zero material.
__global__ void k_prepare_materials(int n, const float *__restrict__ albedo, const int32_t *__restrict__ is_light,
                                    const int32_t *__restrict__ kind, const float *__restrict__ shininess,
                                    float4 *__restrict__ mat, float *__restrict__ shin, float *__restrict__ emission) {
  int const total = n > 0 ? n : 1;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float e = 1.0f;
    if (n > 0) {
      int const k = kind ? kind[m] : XYZGPU_MATERIAL_LAMBERT;
      bool const light = is_light[m] != 0;
      float const kw = light ? 1.0f : (k != XYZGPU_MATERIAL_LAMBERT ? static_cast<float>(k) : 0.0f);
      r = make_float4(albedo[3 * m], albedo[3 * m + 1], albedo[3 * m + 2], kw);
      if (!light && k == XYZGPU_MATERIAL_METAL) e = shininess[m];
    }
    mat[m] = r;
    shin[m] = e;
    emission[m] = 1.0f;
  }
}

__global__ void k_set_materials(float4 *__restrict__ mat, float *__restrict__ emission,
                                const float *__restrict__ albedo_in, const float *__restrict__ emission_in,
                                int nm) {
  int const m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  if (albedo_in) {
    float4 r = mat[m];
    r.x = albedo_in[3 * m];
    r.y = albedo_in[3 * m + 1];
    r.z = albedo_in[3 * m + 2];
    mat[m] = r;
  }
  if (emission_in) emission[m] = emission_in[m];
}

int materials_device_update(SceneImpl &s, const float *albedo_xyz, const float *emission, cudaStream_t st) {
  if (!albedo_xyz && !emission) return XYZGPU_OK;
  int const nm = s.n_materials;
  k_set_materials<<<(nm + 255) / 256, 256, 0, st>>>(s.d_mat, s.d_emission, albedo_xyz, emission, nm);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

}  // namespace
}  // namespace xyzgpu

using namespace xyzgpu;

extern "C" {

int xyzgpu_abi_version(void) { return XYZGPU_ABI_VERSION; }

const char *xyzgpu_last_error(void) { return g_last_error.c_str(); }

float xyzgpu_philox_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t dim) {
  uint32_t w[4];
  philox4x32_10(pixel, sample, dim >> 2, 0u, static_cast<uint32_t>(seed),
                static_cast<uint32_t>(seed >> 32), w);
  return u01_from_bits(w[dim & 3u]);
}

void xyzgpu_build_params_default(xyzgpu_build_params *bp) {
  if (!bp) return;
  // chosen by a sweep on the 1M-triangle benchmark scene and the occluded
  // room (traversal time per frame, build time)
  bp->leaf_max_tris = 8;
  bp->max_depth = 0;
  bp->cost_traversal = 1.0f;
  bp->cost_intersect = 1.5f;
  bp->empty_bonus = 0.0f;
  bp->bins = 64;
  bp->builder = XYZGPU_BUILD_DEVICE;
  bp->max_refs_factor = 6;
}

void xyzgpu_render_params_default(xyzgpu_render_params *rp) {
  if (!rp) return;
  std::memset(rp, 0, sizeof(*rp));
  rp->width = 256;
  rp->height = 256;
  rp->spp = 1;
  rp->spp_offset = 0;
  rp->max_depth = 15;
  rp->rr_start_depth = 1;
  rp->rr_threshold = 0.2f;
  rp->seed = 0;
  rp->film_location = XYZGPU_FILM_DEVICE;
  rp->accumulate = 0;
  rp->wave_paths = 0;
  rp->profile = XYZGPU_PROFILE_OFF;
  rp->spectral = XYZGPU_SPECTRAL_OFF;
  rp->hero_wavelengths = 4;
}

int xyzgpu_scene_create(const xyzgpu_scene_desc *d, const xyzgpu_build_params *bp_in,
                        xyzgpu_scene *out) {
  clear_error();
  if (!d || !out) return set_error(XYZGPU_E_INVALID, "scene_create: null argument");
  *out = nullptr;
  xyzgpu_build_params bp;
  if (bp_in) {
    bp = *bp_in;
  } else {
    xyzgpu_build_params_default(&bp);
  }
  if (d->n_triangles < 0 || d->n_vertices < 0 || d->n_materials < 0)
    return set_error(XYZGPU_E_INVALID, "scene_create: negative count");
  if (d->n_triangles >= (1 << 29))
    return set_error(XYZGPU_E_LIMIT, "scene_create: %d triangles exceeds the limit of 2^29 - 1",
                     d->n_triangles);
  if (d->n_triangles > 0 && (!d->positions || !d->triangles || !d->tri_material))
    return set_error(XYZGPU_E_INVALID, "scene_create: null geometry array");
  if (d->n_materials > 0 && (!d->albedo_xyz || !d->is_light))
    return set_error(XYZGPU_E_INVALID, "scene_create: null material array");
  if (bp.leaf_max_tris < 1 || bp.bins < 2 || bp.bins > kKdMaxBins || bp.max_depth < 0 ||
      bp.max_depth > kKdMaxDepthLimit || !(bp.cost_traversal >= 0) || !(bp.cost_intersect > 0) ||
      !(bp.empty_bonus >= 0 && bp.empty_bonus < 1) || bp.max_refs_factor < 1)
    return set_error(XYZGPU_E_INVALID, "scene_create: build parameters out of range");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(d->light_power_xyz[k]))
      return set_error(XYZGPU_E_INVALID, "scene_create: light power is not finite");
  int dev = 0;
  int rc = check_device(&dev);
  if (rc) return rc;

  int const nt = d->n_triangles, nv = d->n_vertices, nm = d->n_materials;
  bool const smooth = d->normals != nullptr;
  int n_specular = 0;
  for (int m = 0; m < nm; ++m) {
    int const kind = d->material_kind ? d->material_kind[m] : XYZGPU_MATERIAL_LAMBERT;
    if (kind != XYZGPU_MATERIAL_LAMBERT && kind != XYZGPU_MATERIAL_MIRROR && kind != XYZGPU_MATERIAL_METAL)
      return set_error(XYZGPU_E_INVALID, "scene_create: material %d has unknown kind %d", m, kind);
    if (!d->is_light[m] && kind != XYZGPU_MATERIAL_LAMBERT) ++n_specular;
    if (kind == XYZGPU_MATERIAL_METAL && !d->is_light[m]) {
      if (!d->shininess || !(d->shininess[m] > 0.0f) || !std::isfinite(d->shininess[m]))
        return set_error(XYZGPU_E_INVALID, "scene_create: metal material %d needs a shininess > 0", m);
    }
  }
  SceneImpl *s = new (std::nothrow) SceneImpl();
  if (!s) return set_error(XYZGPU_E_NOMEM, "scene_create: host allocation failed");
  s->device = dev;
  s->n_tris = nt;
  s->n_materials = nm;
  s->n_specular = n_specular;
  s->smooth = smooth;
  configure_pool(dev);
  cudaStream_t const st = nullptr;
  int64_t bytes = 0, scratch = 0;
  float *d_pos = nullptr, *d_nrm = nullptr, *d_box = nullptr, *d_alb = nullptr, *d_shin = nullptr;
  int32_t *d_idx = nullptr, *d_tmat = nullptr, *d_lit = nullptr, *d_kind = nullptr, *d_flag = nullptr,
          *d_lid = nullptr;
  int8_t *d_lflag = nullptr;
  uint8_t *d_tmp = nullptr;
  auto free_temps = [&]() {
    cudaFreeAsync(d_flag, st);
    cudaFreeAsync(d_lid, st);
    cudaFreeAsync(d_lflag, st);
    cudaFreeAsync(d_tmp, st);
    d_flag = d_lid = nullptr;
    d_lflag = nullptr;
    d_tmp = nullptr;
    cudaFreeAsync(d_pos, st);
    cudaFreeAsync(d_nrm, st);
    cudaFreeAsync(d_idx, st);
    cudaFreeAsync(d_tmat, st);
    cudaFreeAsync(d_box, st);
    cudaFreeAsync(d_alb, st);
    cudaFreeAsync(d_lit, st);
    cudaFreeAsync(d_kind, st);
    cudaFreeAsync(d_shin, st);
    d_pos = d_nrm = d_box = d_alb = d_shin = nullptr;
    d_idx = d_tmat = d_lit = d_kind = nullptr;
  };
  auto fail = [&](int r) {
    free_temps();
    free_scene(s);
    return r;
  };
#define XYZ_TRY(expr)      \
  do {                     \
    int const r_ = (expr); \
    if (r_) return fail(r_); \
  } while (0)
  XYZ_TRY(dev_upload(&d_pos, d->positions, 3 * static_cast<size_t>(nv), &scratch, st));
  if (smooth) XYZ_TRY(dev_upload(&d_nrm, d->normals, 3 * static_cast<size_t>(nv), &scratch, st));
  XYZ_TRY(dev_upload(&d_idx, d->triangles, 3 * static_cast<size_t>(nt), &scratch, st));
  XYZ_TRY(dev_upload(&d_tmat, d->tri_material, static_cast<size_t>(nt), &scratch, st));
  XYZ_TRY(dev_alloc(&s->d_tri, 3 * static_cast<size_t>(nt), &bytes, st));
  XYZ_TRY(dev_alloc(&s->d_ng, static_cast<size_t>(nt), &bytes, st));
  if (smooth) XYZ_TRY(dev_alloc(&s->d_sn, 3 * static_cast<size_t>(nt), &bytes, st));
  // the material table is built on the device from the caller's arrays
  // (copies of caller memory are fast; a table assembled in freshly
  // allocated host memory uploads several times slower)
  {
    size_t const nmat = nm > 0 ? static_cast<size_t>(nm) : 1;
    XYZ_TRY(dev_alloc(&s->d_mat, nmat, &bytes, st));
    XYZ_TRY(dev_alloc(&s->d_shininess, nmat, &bytes, st));
    XYZ_TRY(dev_alloc(&s->d_emission, nmat, &bytes, st));
    if (nm > 0) {
      XYZ_TRY(dev_upload(&d_alb, d->albedo_xyz, 3 * static_cast<size_t>(nm), &scratch, st));
      XYZ_TRY(dev_upload(&d_lit, d->is_light, static_cast<size_t>(nm), &scratch, st));
      if (d->material_kind) XYZ_TRY(dev_upload(&d_kind, d->material_kind, static_cast<size_t>(nm), &scratch, st));
      if (d->shininess) XYZ_TRY(dev_upload(&d_shin, d->shininess, static_cast<size_t>(nm), &scratch, st));
    }
    k_prepare_materials<<<static_cast<int>(std::min<size_t>((nmat + 255) / 256, 4096)), 256, 0, st>>>(
        nm, d_alb, d_lit, d_kind, d_shin, s->d_mat, s->d_shininess, s->d_emission);
    cudaError_t const e = cudaGetLastError();
    if (e != cudaSuccess) return fail(set_error(XYZGPU_E_CUDA, "scene_create: %s", cudaGetErrorString(e)));
  }
  if (d->albedo_spd) XYZ_TRY(dev_upload(&s->d_spd, d->albedo_spd, 31 * static_cast<size_t>(nm), &bytes, st));
  XYZ_TRY(dev_alloc(&s->d_fetch, 64, &bytes, st));
  XYZ_TRY(dev_alloc(&s->d_trace_counts, 8, &bytes, st));
  XYZ_TRY(dev_alloc(&d_box, 6, &scratch, st));
  float const box_init[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  if (cudaMemcpyAsync(d_box, box_init, sizeof(box_init), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return fail(set_error(XYZGPU_E_CUDA, "scene_create: copy failed"));
  // checks of the caller's geometry on the device (finite coordinates,
  // indices in range) and the light triangles in triangle order
  XYZ_TRY(dev_alloc(&d_flag, 2, &scratch, st));
  XYZ_TRY(dev_alloc(&d_lflag, static_cast<size_t>(nt), &scratch, st));
  XYZ_TRY(dev_alloc(&d_lid, static_cast<size_t>(nt), &scratch, st));
  if (cudaMemsetAsync(d_flag, 0, 2 * sizeof(int), st) != cudaSuccess)
    return fail(set_error(XYZGPU_E_CUDA, "scene_create: memset failed"));
  if (nv > 0) k_check_finite<<<static_cast<int>(std::min<int64_t>((3ll * nv + 255) / 256, 2048)), 256, 0, st>>>(
      d_pos, 3ll * nv, d_flag);
  if (nt > 0) {
    k_prepare_triangles<<<(nt + 255) / 256, 256, 0, st>>>(d_pos, d_nrm, d_idx, d_tmat, nt, nv, nm, d_lit, s->d_tri,
                                                           s->d_ng, s->d_sn, d_box, d_box + 3, d_flag, d_lflag);
    size_t tmp_bytes = 0;
    thrust::counting_iterator<int32_t> ids(0);
    if (cub::DeviceSelect::Flagged(nullptr, tmp_bytes, ids, d_lflag, d_lid, d_flag + 1, nt, st) != cudaSuccess)
      return fail(set_error(XYZGPU_E_CUDA, "scene_create: light selection failed"));
    XYZ_TRY(dev_alloc(&d_tmp, tmp_bytes, &scratch, st));
    if (cub::DeviceSelect::Flagged(d_tmp, tmp_bytes, ids, d_lflag, d_lid, d_flag + 1, nt, st) != cudaSuccess)
      return fail(set_error(XYZGPU_E_CUDA, "scene_create: light selection failed"));
    cudaError_t const e = cudaGetLastError();
    if (e != cudaSuccess) return fail(set_error(XYZGPU_E_CUDA, "scene_create: %s", cudaGetErrorString(e)));
  }
  float box[6];
  int flags[2] = {0, 0};
  if (cudaMemcpyAsync(box, d_box, sizeof(box), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(flags, d_flag, sizeof(flags), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail(set_error(XYZGPU_E_CUDA, "scene_create: triangle preparation failed"));
  if (flags[0]) return fail(host_geometry_error(d));
  // light CDF in triangle order (xyz/core/scene_mqo.cpp:512-519), with the
  // area of Triangle::area (xyz/geom/triangle.hpp:57-59)
  std::vector<int32_t> lights(static_cast<size_t>(nt > 0 ? flags[1] : 0));
  if (!lights.empty() && cudaMemcpy(lights.data(), d_lid, lights.size() * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(set_error(XYZGPU_E_CUDA, "scene_create: reading the light list failed"));
  std::vector<float> cdf(1, 0.0f);
  cdf.reserve(lights.size() + 1);
  for (int32_t const i : lights) {
    int32_t const a = d->triangles[3 * i], b = d->triangles[3 * i + 1], c = d->triangles[3 * i + 2];
    f3 const p0 = mk3(d->positions[3 * a], d->positions[3 * a + 1], d->positions[3 * a + 2]);
    f3 const p1 = mk3(d->positions[3 * b], d->positions[3 * b + 1], d->positions[3 * b + 2]);
    f3 const p2 = mk3(d->positions[3 * c], d->positions[3 * c + 1], d->positions[3 * c + 2]);
    f3 const n = cross3(sub3(p2, p0), sub3(p1, p0));
    float const area = std::sqrt(dot3(n, n)) * 0.5f;
    cdf.push_back(cdf.back() + area);
  }
  s->n_lights = static_cast<int>(lights.size());
  XYZ_TRY(dev_upload(&s->d_lights, lights.data(), lights.size(), &bytes, st));
  XYZ_TRY(dev_upload(&s->d_cdf, cdf.data(), cdf.size(), &bytes, st));
  free_temps();
#undef XYZ_TRY
  // root box: the bounds grown by 1e-5 of the extent plus 1e-6 (kd_root_bounds)
  for (int k = 0; k < 3; ++k) {
    float lo = box[k], hi = box[3 + k];
    if (nt == 0) lo = hi = 0.0f;
    float const pad = (hi - lo) * 1e-5f + 1e-6f;
    box[k] = lo - pad;
    box[3 + k] = hi + pad;
  }
  s->dev.bmin = mk3(box[0], box[1], box[2]);
  s->dev.bmax = mk3(box[3], box[4], box[5]);

  BuildConfig cfg;
  cfg.leaf_max_tris = bp.leaf_max_tris;
  cfg.max_depth = kd_resolve_max_depth(bp.max_depth, nt);
  cfg.cost_traversal = bp.cost_traversal;
  cfg.cost_intersect = bp.cost_intersect;
  cfg.empty_bonus = bp.empty_bonus;
  cfg.bins = bp.bins;
  cfg.max_refs = static_cast<int64_t>(bp.max_refs_factor) * nt + 1024;
  auto const t0 = std::chrono::steady_clock::now();
  if (bp.builder == XYZGPU_BUILD_HOST) {
    // the host builder reads the triangles' vertices back from the device
    std::vector<float4> tri(3 * static_cast<size_t>(nt));
    if (nt && cudaMemcpy(tri.data(), s->d_tri, tri.size() * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess) {
      free_scene(s);
      return set_error(XYZGPU_E_CUDA, "scene_create: reading triangles back failed");
    }
    std::vector<float> trv(9 * static_cast<size_t>(nt));
    for (int i = 0; i < nt; ++i) {
      f3 const p0 = xyz3(tri[3 * i]), e1 = xyz3(tri[3 * i + 1]), e2 = xyz3(tri[3 * i + 2]);
      f3 const q1 = add3(p0, e1), q2 = add3(p0, e2);
      float *tv = &trv[9 * static_cast<size_t>(i)];
      tv[0] = p0.x, tv[1] = p0.y, tv[2] = p0.z;
      tv[3] = q1.x, tv[4] = q1.y, tv[5] = q1.z;
      tv[6] = q2.x, tv[7] = q2.y, tv[8] = q2.z;
    }
    KdTreeHost tree;
    std::string err;
    if (!kd_build_host(trv.data(), nt, cfg, &tree, &err)) {
      free_scene(s);
      return set_error(XYZGPU_E_LIMIT, "scene_create: %s", err.c_str());
    }
    s->n_nodes = static_cast<int64_t>(tree.nodes.size() / 2);
    s->n_refs = static_cast<int64_t>(tree.refs.size());
    s->n_leaves = tree.leaves;
    s->n_empty = tree.empty_leaves;
    s->depth = tree.depth;
    std::vector<uint2> nodes(s->n_nodes);
    for (int64_t j = 0; j < s->n_nodes; ++j) nodes[j] = make_uint2(tree.nodes[2 * j], tree.nodes[2 * j + 1]);
    int r2 = dev_upload(&s->d_nodes, nodes.data(), nodes.size(), &bytes, st);
    if (!r2) r2 = dev_upload(&s->d_refs, tree.refs.data(), tree.refs.size(), &bytes, st);
    if (!r2) {
      // level ranges of the breadth-first array: each level's interior nodes
      // own the next level's child pairs
      std::vector<int64_t> level_start{0};
      int64_t b = 0, e = s->n_nodes > 0 ? 1 : 0;
      while (e > b) {
        level_start.push_back(e);
        int64_t interior = 0;
        for (int64_t j = b; j < e; ++j) interior += (nodes[j].y & 3u) != kKdLeafTag;
        b = e;
        e = b + 2 * interior;
      }
      if (s->n_nodes > 0) r2 = kd_layout_depth_first(*s, level_start, st);
    }
    if (r2) {
      free_scene(s);
      return r2;
    }
  } else if (bp.builder == XYZGPU_BUILD_DEVICE) {
    int r2 = kd_build_device(*s, s->d_tri, nt, cfg, st);
    if (r2) {
      free_scene(s);
      return r2;
    }
    bytes += s->n_nodes * 8 + s->n_refs * 4;
  } else {
    free_scene(s);
    return set_error(XYZGPU_E_INVALID, "scene_create: unknown builder %d", bp.builder);
  }
  s->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  s->device_bytes = bytes;

  DevScene &v = s->dev;
  v.tri = s->d_tri;
  v.tri_ng = s->d_ng;
  v.tri_sn = s->d_sn;
  v.mat = s->d_mat;
  v.shininess = s->d_shininess;
  v.has_metal = 0;
  if (d->material_kind)
    for (int m = 0; m < nm; ++m)
      if (!d->is_light[m] && d->material_kind[m] == XYZGPU_MATERIAL_METAL) v.has_metal = 1;
  v.emission = s->d_emission;
  v.lights = s->d_lights;
  v.cdf = s->d_cdf;
  v.nodes = s->d_nodes;
  v.refs = s->d_refs;
  // Lights of zero total area cannot be sampled: next-event estimation is off
  // (the reference would divide by that area, xyz/core/scene.cpp:65).
  v.n_lights = cdf.back() > 0.0f ? s->n_lights : 0;
  v.light_area = cdf.back();
  v.power = mk3(d->light_power_xyz[0], d->light_power_xyz[1], d->light_power_xyz[2]);
  v.spd_albedo = s->d_spd;
  for (int i = 0; i < 31; ++i) v.spd_light[i] = d->albedo_spd ? d->light_power_spd[i] : 0.0f;
  cudaError_t const e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    free_scene(s);
    return set_error(XYZGPU_E_CUDA, "scene_create: %s", cudaGetErrorString(e));
  }
  *out = reinterpret_cast<xyzgpu_scene>(s);
  return XYZGPU_OK;
}

void xyzgpu_scene_destroy(xyzgpu_scene scene) { free_scene(reinterpret_cast<SceneImpl *>(scene)); }

int xyzgpu_scene_stats_get(xyzgpu_scene scene, xyzgpu_scene_stats *o) {
  clear_error();
  if (!scene || !o) return set_error(XYZGPU_E_INVALID, "scene_stats_get: null argument");
  SceneImpl const *s = reinterpret_cast<SceneImpl *>(scene);
  o->n_triangles = s->n_tris;
  o->n_lights = s->n_lights;
  o->n_nodes = s->n_nodes;
  o->n_leaves = s->n_leaves;
  o->n_empty_leaves = s->n_empty;
  o->n_leaf_refs = s->n_refs;
  o->max_depth = s->depth;
  o->device_bytes = s->device_bytes;
  o->build_ms = s->build_ms;
  o->light_area = s->dev.light_area;
  o->bounds_min[0] = s->dev.bmin.x, o->bounds_min[1] = s->dev.bmin.y, o->bounds_min[2] = s->dev.bmin.z;
  o->bounds_max[0] = s->dev.bmax.x, o->bounds_max[1] = s->dev.bmax.y, o->bounds_max[2] = s->dev.bmax.z;
  return XYZGPU_OK;
}

int xyzgpu_scene_copy_tree(xyzgpu_scene scene, uint32_t *nodes, int32_t *refs) {
  clear_error();
  if (!scene) return set_error(XYZGPU_E_INVALID, "scene_copy_tree: null scene");
  SceneImpl const *s = reinterpret_cast<SceneImpl *>(scene);
  if (nodes && s->n_nodes)
    XYZ_CUDA_TRY(cudaMemcpy(nodes, s->d_nodes, s->n_nodes * 8, cudaMemcpyDeviceToHost));
  if (refs && s->n_refs)
    XYZ_CUDA_TRY(cudaMemcpy(refs, s->d_refs, s->n_refs * 4, cudaMemcpyDeviceToHost));
  return XYZGPU_OK;
}

int xyzgpu_trace_closest(xyzgpu_scene scene, const float *rays, int n, float *hits, void *stream) {
  clear_error();
  if (!scene) return set_error(XYZGPU_E_INVALID, "trace_closest: null scene");
  if (n < 0) return set_error(XYZGPU_E_INVALID, "trace_closest: negative ray count");
  if (n > 0 && (!rays || !hits)) return set_error(XYZGPU_E_INVALID, "trace_closest: null buffer");
  if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u)
    return set_error(XYZGPU_E_INVALID, "trace_closest: buffers must be 16-byte aligned");
  return trace_api_launch(*reinterpret_cast<SceneImpl *>(scene), rays, n, hits,
                          static_cast<cudaStream_t>(stream), nullptr);
}

int xyzgpu_trace_closest_counted(xyzgpu_scene scene, const float *rays, int n, float *hits,
                                 void *stream, xyzgpu_trace_counters *counters) {
  clear_error();
  if (!scene || !counters) return set_error(XYZGPU_E_INVALID, "trace_closest_counted: null argument");
  if (n < 0) return set_error(XYZGPU_E_INVALID, "trace_closest_counted: negative ray count");
  if (n > 0 && (!rays || !hits)) return set_error(XYZGPU_E_INVALID, "trace_closest_counted: null buffer");
  if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u)
    return set_error(XYZGPU_E_INVALID, "trace_closest_counted: buffers must be 16-byte aligned");
  return trace_api_launch(*reinterpret_cast<SceneImpl *>(scene), rays, n, hits,
                          static_cast<cudaStream_t>(stream), counters);
}

}  // extern "C"

namespace xyzgpu {
// Checks shared by xyzgpu_render, xyzgpu_adjoint and xyzgpu_render_importon.
int check_render_args(const char *who, xyzgpu_scene scene, const xyzgpu_camera *cam,
                      const xyzgpu_render_params *rp) {
  if (rp->width <= 0 || rp->height <= 0 || rp->spp < 0 || rp->spp_offset < 0 ||
      rp->max_depth < 1 || rp->max_depth > 1000 || rp->rr_start_depth < 1 ||
      !(rp->rr_threshold >= 0.0f) || rp->wave_paths < 0 || rp->profile < 0 || rp->profile > 2 ||
      rp->spectral < 0 || rp->spectral > 2 ||
      (rp->spectral && (rp->hero_wavelengths < 1 || rp->hero_wavelengths > 4)) ||
      (rp->film_location != XYZGPU_FILM_DEVICE && rp->film_location != XYZGPU_FILM_HOST) ||
      !((rp->row_begin == 0 && rp->row_end == 0) ||
        (rp->row_begin >= 0 && rp->row_begin < rp->row_end && rp->row_end <= rp->height)) ||
      rp->row_step < 0)
    return set_error(XYZGPU_E_INVALID, "%s: parameters out of range", who);
  if (static_cast<int64_t>(rp->width) * rp->height >= (1ll << 31))
    return set_error(XYZGPU_E_LIMIT, "%s: image of %d x %d pixels exceeds 2^31", who, rp->width,
                     rp->height);
  if (static_cast<int64_t>(rp->spp_offset) + rp->spp >= (1ll << 32))
    return set_error(XYZGPU_E_LIMIT, "%s: sample index exceeds 2^32", who);
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(cam->eye[k]) || !std::isfinite(cam->at[k]))
      return set_error(XYZGPU_E_INVALID, "%s: camera position is not finite", who);
  if (!(cam->film_size > 0) || !(cam->focal_length > 0) || !(cam->f_number > 0))
    return set_error(XYZGPU_E_INVALID, "%s: camera film size, focal length and F-number must be > 0", who);
  if (rp->spectral && reinterpret_cast<SceneImpl *>(scene)->n_specular)
    return set_error(XYZGPU_E_INVALID, "%s: mirror and metal materials render in the XYZ film mode only", who);
  if (rp->spectral && !reinterpret_cast<SceneImpl *>(scene)->d_spd)
    return set_error(XYZGPU_E_INVALID, "%s: the spectral film modes need albedo spectra in the scene", who);
  return XYZGPU_OK;
}
}  // namespace xyzgpu

extern "C" {

int xyzgpu_render(xyzgpu_scene scene, const xyzgpu_camera *cam, const xyzgpu_render_params *rp,
                  float *film, void *stream) {
  clear_error();
  if (!scene || !cam || !rp || !film) return set_error(XYZGPU_E_INVALID, "render: null argument");
  int const rc = check_render_args("render", scene, cam, rp);
  if (rc) return rc;
  return render_launch(*reinterpret_cast<SceneImpl *>(scene), *cam, *rp, film,
                       static_cast<cudaStream_t>(stream));
}

int xyzgpu_adjoint(xyzgpu_scene scene, const xyzgpu_camera *cam, const xyzgpu_render_params *rp,
                   const float *d_film, float *d_albedo, float *d_emission, void *stream) {
  clear_error();
  if (!scene || !cam || !rp || !d_film || !d_albedo || !d_emission)
    return set_error(XYZGPU_E_INVALID, "adjoint: null argument");
  int const rc = check_render_args("adjoint", scene, cam, rp);
  if (rc) return rc;
  if (rp->spectral != XYZGPU_SPECTRAL_OFF)
    return set_error(XYZGPU_E_INVALID, "adjoint: only the XYZ film mode is differentiated");
  if (reinterpret_cast<SceneImpl *>(scene)->n_specular)
    return set_error(XYZGPU_E_INVALID, "adjoint: scenes with mirror or metal materials are not differentiated");
  if (rp->profile != XYZGPU_PROFILE_OFF)
    return set_error(XYZGPU_E_INVALID, "adjoint: profiling is not supported");
  if ((reinterpret_cast<uintptr_t>(d_film) | reinterpret_cast<uintptr_t>(d_albedo) |
       reinterpret_cast<uintptr_t>(d_emission)) & 3u)
    return set_error(XYZGPU_E_INVALID, "adjoint: buffers must be 4-byte aligned");
  AdjointArgs adj{d_film, d_albedo, d_emission};
  return render_launch(*reinterpret_cast<SceneImpl *>(scene), *cam, *rp, nullptr,
                       static_cast<cudaStream_t>(stream), &adj);
}

int xyzgpu_scene_set_materials(xyzgpu_scene scene, const float *albedo_xyz, const float *emission,
                               int location, void *stream) {
  clear_error();
  if (!scene) return set_error(XYZGPU_E_INVALID, "scene_set_materials: null scene");
  if (location != XYZGPU_FILM_DEVICE && location != XYZGPU_FILM_HOST)
    return set_error(XYZGPU_E_INVALID, "scene_set_materials: unknown location %d", location);
  SceneImpl &s = *reinterpret_cast<SceneImpl *>(scene);
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  int const nm = s.n_materials;
  if (nm == 0) return XYZGPU_OK;
  if (location == XYZGPU_FILM_HOST) {
    // host values are checked and copied synchronously
    if (albedo_xyz) {
      std::vector<float4> mat(nm);
      XYZ_CUDA_TRY(cudaMemcpyAsync(mat.data(), s.d_mat, nm * sizeof(float4), cudaMemcpyDeviceToHost, st));
      XYZ_CUDA_TRY(cudaStreamSynchronize(st));
      for (int m = 0; m < nm; ++m) {
        for (int c = 0; c < 3; ++c)
          if (!std::isfinite(albedo_xyz[3 * m + c]))
            return set_error(XYZGPU_E_INVALID, "scene_set_materials: albedo of material %d is not finite", m);
        mat[m].x = albedo_xyz[3 * m];
        mat[m].y = albedo_xyz[3 * m + 1];
        mat[m].z = albedo_xyz[3 * m + 2];
      }
      XYZ_CUDA_TRY(cudaMemcpyAsync(s.d_mat, mat.data(), nm * sizeof(float4), cudaMemcpyHostToDevice, st));
      XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (emission) {
      for (int m = 0; m < nm; ++m)
        if (!std::isfinite(emission[m]))
          return set_error(XYZGPU_E_INVALID, "scene_set_materials: emission of material %d is not finite", m);
      XYZ_CUDA_TRY(cudaMemcpyAsync(s.d_emission, emission, nm * sizeof(float), cudaMemcpyHostToDevice, st));
      XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return XYZGPU_OK;
  }
  return materials_device_update(s, albedo_xyz, emission, st);
}

int xyzgpu_scene_get_materials(xyzgpu_scene scene, float *albedo_xyz, float *emission) {
  clear_error();
  if (!scene) return set_error(XYZGPU_E_INVALID, "scene_get_materials: null scene");
  SceneImpl &s = *reinterpret_cast<SceneImpl *>(scene);
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  int const nm = s.n_materials;
  if (nm == 0) return XYZGPU_OK;
  if (albedo_xyz) {
    std::vector<float4> mat(nm);
    XYZ_CUDA_TRY(cudaMemcpy(mat.data(), s.d_mat, nm * sizeof(float4), cudaMemcpyDeviceToHost));
    for (int m = 0; m < nm; ++m) {
      albedo_xyz[3 * m] = mat[m].x;
      albedo_xyz[3 * m + 1] = mat[m].y;
      albedo_xyz[3 * m + 2] = mat[m].z;
    }
  }
  if (emission) XYZ_CUDA_TRY(cudaMemcpy(emission, s.d_emission, nm * sizeof(float), cudaMemcpyDeviceToHost));
  return XYZGPU_OK;
}

int xyzgpu_render_noalloc(xyzgpu_scene scene, const xyzgpu_camera *cam,
                          const xyzgpu_render_params *rp, float *film, void *stream) {
  clear_error();
  if (!scene || !cam || !rp || !film) return set_error(XYZGPU_E_INVALID, "render_noalloc: null argument");
  if (rp->width <= 0 || rp->height <= 0 || rp->spp < 0 || rp->spp_offset < 0 ||
      rp->max_depth < 1 || rp->rr_start_depth < 1 || !(rp->rr_threshold >= 0.0f) ||
      rp->wave_paths < 0 || rp->row_begin != 0 || rp->row_end != 0)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: parameters out of range (row bands are not available)");
  if (static_cast<int64_t>(rp->width) * rp->height >= (1ll << 31))
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: image of %d x %d pixels exceeds 2^31",
                     rp->width, rp->height);
  if (static_cast<int64_t>(rp->spp_offset) + rp->spp >= (1ll << 32))
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: sample index exceeds 2^32");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(cam->eye[k]) || !std::isfinite(cam->at[k]))
      return set_error(XYZGPU_E_INVALID, "render_noalloc: camera position is not finite");
  if (!(cam->film_size > 0) || !(cam->focal_length > 0) || !(cam->f_number > 0))
    return set_error(XYZGPU_E_INVALID,
                     "render_noalloc: camera film size, focal length and F-number must be > 0");
  if (reinterpret_cast<uintptr_t>(film) & 3u)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: film must be 4-byte aligned");
  return render_noalloc_launch(*reinterpret_cast<SceneImpl *>(scene), *cam, *rp, film,
                               static_cast<cudaStream_t>(stream));
}

int xyzgpu_render_counters_get(xyzgpu_scene scene, xyzgpu_render_counters *out) {
  clear_error();
  if (!scene || !out) return set_error(XYZGPU_E_INVALID, "render_counters_get: null argument");
  SceneImpl &s = *reinterpret_cast<SceneImpl *>(scene);
  int const rc = render_collect(s);
  if (rc) return rc;
  *out = s.counters;
  return XYZGPU_OK;
}

int xyzgpu_render_profile_get(xyzgpu_scene scene, xyzgpu_render_profile *out) {
  clear_error();
  if (!scene || !out) return set_error(XYZGPU_E_INVALID, "render_profile_get: null argument");
  SceneImpl &s = *reinterpret_cast<SceneImpl *>(scene);
  int const rc = render_collect(s);
  if (rc) return rc;
  *out = s.profile;
  return XYZGPU_OK;
}

}  // extern "C"
