// Importance-driven path tracing on the GPU: the reference's non-learned
// path guide (Scene::EvaluteImportanceDrivenPathTracing, xyz/core/
// scene_importancedrivenpathtracing.cpp:11-180) with its light-importance map
// (Scene::CreateLightImportanceMap, xyz/core/scene_photonmap.cpp:272-330) and
// histogram query (ImportanceQuery, xyz/core/photonmap.cpp:321-439).
//
// Map: light particles are traced as a small wavefront (closest hit with the
// persistent traversal, then a bounce kernel); every Lambert hit from bounce
// `min_depth` on leaves an importon (hit point, incoming direction).  The
// importons are sorted into a uniform grid of cells no smaller than the
// search radius (a counting sort), so a query reads the 27 cells around its
// point: the same set the reference's kd-tree range search finds.
//
// Rendering: after each extension trace of the guided bounces,
// k_importon_query builds each queue entry's 16-bin (cos^2 theta, phi)
// histogram about its shading frame (cumulative counts, 64 B per entry); the
// shading kernel samples directions from it and weights next-event
// estimation with its density (k_shade<kModeImporton>).
//
// As the variants that act in Lambert-only scenes: importons at every Lambert
// hit from bounce min_depth (the source's commented `depth > 0` test; its
// active test also wants a specular bounce first) and histogram sampling at
// every Lambert vertex of the first guide_bounces (its "[TEST]" condition).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "wavefront.cuh"

namespace xyzgpu {

struct ImportonImpl {
  SceneImpl *scene = nullptr;
  int device = 0;
  xyzgpu_importon_config cfg{};
  int64_t n = 0;              // importons in the map
  float4 *d_pos = nullptr;    // sorted by cell: (position, 0)
  float4 *d_dir = nullptr;    //                 (incoming direction, 0)
  int32_t *d_start = nullptr; // cells + 1 prefix offsets
  float3 lo{};                // grid origin
  float cs = 1.0f;            // cell size (>= radius)
  int g[3] = {1, 1, 1};
  float *d_cdf = nullptr;     // per extension-queue entry: 16 cumulative counts
  int64_t cdf_cap = 0;
};

namespace {

constexpr int kImpThreads = 256;

int grid1(int device, int64_t n, int per_sm = 8) {
  int64_t const want = (n + kImpThreads - 1) / kImpThreads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count(device)) * per_sm)));
}

// The uniform grid as the kernels see it.
struct ImpGrid {
  const float4 *pos, *dir;
  const int32_t *start;
  float3 lo;
  float cs, r2;
  int g0, g1, g2;
};

XYZ_DEV int cell_of(float v, float lo, float cs, int g) {
  int const c = static_cast<int>(floorf((v - lo) / cs));
  return c < 0 ? 0 : (c >= g ? g - 1 : c);
}

// ---------------------------------------------------------------- particles
// Particle p reads the Philox stream (pixel = p, sample = 0xffffffff): the
// light point (two draws, as SampleLightPosition), a cosine direction about
// the light's geometric normal (two draws), then per Lambert hit one roulette
// draw (survival albedo.y, Lambert::BoundsImportance, xyz/bsdf/lambert.cpp:
// 16-42) and two for the next cosine direction about the hit's geometric
// normal (Triangle::GeometricBasis frame, xyz/geom/triangle.cpp:167-192).
constexpr uint32_t kParticleSample = 0xffffffffu;

XYZ_DEV void frame_about(f3 n, f3 *t, f3 *b) {
  f3 tt = mk3(-n.z, 0.0f, n.x);
  float const l2 = dot3(tt, tt);
  if (l2 > 0.0f) {
    tt = scl3(tt, 1.0f / sqrtf(l2));
    *b = cross3(tt, n);
  } else {
    *b = mk3(0.0f, 0.0f, (n.y > 0.0f) ? 1.0f : -1.0f);
    tt = cross3(n, *b);
  }
  *t = tt;
}

XYZ_DEV f3 cosine_dir(f3 t, f3 b, f3 n, float mu_phi, float mu_theta) {
  float const phi = static_cast<float>(2.0 * kPi) * mu_phi;
  float const cos_t = sqrtf(mu_theta), sin_t = sqrtf(1.0f - mu_theta);
  return add3(add3(scl3(t, sin_t * cosf(phi)), scl3(b, sin_t * sinf(phi))), scl3(n, cos_t));
}

struct ParticleQueue {
  float4 *o, *d;       // ray origin (w: tmin), direction (w: tmax)
  int32_t *pid;        // particle index
  uint32_t *dim;       // next stream dimension
};

__global__ void k_particles_start(DevScene S, int particles, uint64_t seed, ParticleQueue q, int32_t *count) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < particles; p += gridDim.x * blockDim.x) {
    PathRng rng;
    rng.init(seed, static_cast<uint32_t>(p), kParticleSample, 0u);
    float const lt = rng.next();
    float const ls = rng.next();
    // SampleLightPosition + Triangle::Sample (scene.cpp:42-78, triangle.cpp:232-263)
    float const u = ls * __ldg(&S.cdf[S.n_lights]);
    int lo = 0, hi = S.n_lights + 1;
    while (lo < hi) {
      int const mid = (lo + hi) >> 1;
      if (!(u < __ldg(&S.cdf[mid])))
        lo = mid + 1;
      else
        hi = mid;
    }
    int const n = min(max(lo - 1, 0), S.n_lights - 1);
    float const c0 = __ldg(&S.cdf[n]), c1 = __ldg(&S.cdf[n + 1]);
    float const v = (u - c0) / (c1 - c0);
    int32_t const li = __ldg(&S.lights[n]);
    float const ss = sqrtf(v);
    float const uu = ss * (1.0f - lt), vv = ss * lt;
    float4 const a = __ldg(&S.tri[3 * li]), b = __ldg(&S.tri[3 * li + 1]), c = __ldg(&S.tri[3 * li + 2]);
    f3 const pos = add3(add3(xyz3(a), scl3(xyz3(b), uu)), scl3(xyz3(c), vv));
    f3 const gn = xyz3(__ldg(&S.tri_ng[li]));
    f3 t, bb;
    frame_about(gn, &t, &bb);
    float const mp = rng.next();
    float const mt = rng.next();
    f3 const dir = cosine_dir(t, bb, gn, mp, mt);
    q.o[p] = make_float4(pos.x, pos.y, pos.z, kRayTMin);
    q.d[p] = make_float4(dir.x, dir.y, dir.z, __int_as_float(0x7f800000));
    q.pid[p] = p;
    q.dim[p] = rng.dim;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = particles;
}

__global__ void __launch_bounds__(kThreads, 10)
    k_particles_trace(DevScene S, const float4 *qo, const float4 *qd, float4 *hits, const int32_t *count,
                      int32_t *fetch) {
  ExtSink<false> sink{qo, qd, hits, nullptr};
  TraceCount tc{};
  trace_persistent<false>(S, *count, fetch, sink, tc);
}

// One bounce of every live particle: the importon of a Lambert hit from bounce
// min_depth on, then Lambert::BoundsImportance (roulette on albedo.y and a
// cosine direction about the geometric normal).  Lights end the particle
// (Light::BoundsImportance, xyz/bsdf/light.cpp:11-16).
__global__ void k_particles_bounce(DevScene S, int depth, int min_depth, uint64_t seed, ParticleQueue in,
                                   const float4 *hits, const int32_t *count, ParticleQueue out, int32_t *count_out,
                                   float4 *imp_pos, float4 *imp_dir, unsigned long long *n_imp, int64_t imp_cap) {
  int const n = *count;
  int const warp_base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31;
  int const stride = gridDim.x * blockDim.x;
  for (int base = warp_base; base < n; base += stride) {
    int const i = base + (threadIdx.x & 31);
    bool push = false;
    float4 no{}, nd{};
    int32_t pid = 0;
    uint32_t dim = 0;
    if (i < n) {
      float4 const h = hits[i];
      int32_t const code = __float_as_int(h.w);
      if (code >= 0) {
        int32_t const tri = code >> 1;
        int const back = code & 1;
        float4 const g4 = __ldg(&S.tri_ng[tri]);
        int32_t const m = __float_as_int(g4.w);
        if (__ldg(&S.mat[m]).w == 0.0f) {
          float4 const o4 = in.o[i], d4 = in.d[i];
          f3 const d = xyz3(d4);
          f3 gn = xyz3(g4), sn;
          if (S.tri_sn) {
            f3 const n0 = xyz3(__ldg(&S.tri_sn[3 * tri])), s1 = xyz3(__ldg(&S.tri_sn[3 * tri + 1])),
                     s2 = xyz3(__ldg(&S.tri_sn[3 * tri + 2]));
            sn = normalize3(add3(add3(n0, scl3(s1, h.y)), scl3(s2, h.z)));
          } else {
            f3 const z = mk3(0.0f, 0.0f, 0.0f);
            sn = normalize3(add3(add3(gn, scl3(z, h.y)), scl3(z, h.z)));
          }
          if (back) {
            gn = neg3(gn);
            sn = neg3(sn);
          }
          f3 const pos = add3(xyz3(o4), scl3(d, h.x));
          if (depth >= min_depth) {
            unsigned long long const j = atomicAdd(n_imp, 1ull);
            if (static_cast<int64_t>(j) < imp_cap) {
              imp_pos[j] = make_float4(pos.x, pos.y, pos.z, 0.0f);
              imp_dir[j] = make_float4(d.x, d.y, d.z, 0.0f);
            }
          }
          if (!(-dot3(d, sn) <= 0.0f)) {
            pid = in.pid[i];
            PathRng rng;
            rng.init(seed, static_cast<uint32_t>(pid), kParticleSample, in.dim[i]);
            if (!(rng.next() >= __ldg(&S.mat[m]).y)) {
              f3 t, b;
              frame_about(gn, &t, &b);
              float const mp = rng.next();
              float const mt = rng.next();
              f3 const dir = cosine_dir(t, b, gn, mp, mt);
              no = make_float4(pos.x, pos.y, pos.z, kRayTMin);
              nd = make_float4(dir.x, dir.y, dir.z, __int_as_float(0x7f800000));
              dim = rng.dim;
              push = true;
            }
          }
        }
      }
    }
    int32_t const j = warp_append(count_out, push);
    if (push) {
      out.o[j] = no;
      out.d[j] = nd;
      out.pid[j] = pid;
      out.dim[j] = dim;
    }
  }
}

// ---------------------------------------------------------------- grid
__global__ void k_imp_count(const float4 *pos, int64_t n, float3 lo, float cs, int g0, int g1, int g2,
                            int32_t *key, int32_t *cell_count) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float4 const p = pos[i];
    int const c = (cell_of(p.z, lo.z, cs, g2) * g1 + cell_of(p.y, lo.y, cs, g1)) * g0 + cell_of(p.x, lo.x, cs, g0);
    key[i] = c;
    atomicAdd(&cell_count[c], 1);
  }
}

__global__ void k_imp_scatter(const float4 *pos, const float4 *dir, int64_t n, const int32_t *key, int32_t *fill,
                              float4 *pos_out, float4 *dir_out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t const j = atomicAdd(&fill[key[i]], 1);
    pos_out[j] = pos[i];
    dir_out[j] = dir[i];
  }
}

// ---------------------------------------------------------------- query
// begin_query / push_back / end_query (photonmap.cpp:321-373) over the
// importons within the radius of `pos`: 16 bins start at 16 counts; an
// importon counts if it arrives from above the shading normal and its point,
// moved along its direction onto the tangent plane, lies within the radius.
// Writes the cumulative counts c[1..16].
// One query's histogram, computed by a whole warp: the lanes stride over the
// importons of the cells around `pos` (consecutive lanes read consecutive
// importons), each puts its importon in a bin, and 16 ballots per round count
// the bins (lane k keeps bin k).  Every bin starts at 16 counts; lanes 0..15
// return the cumulative counts (integers, exact in float below 2^24).  All
// lanes of the warp call this with the same query.
XYZ_DEV float importon_histogram_warp(const ImpGrid &M, f3 pos, f3 sn, f3 tan, f3 bin, int lane) {
  unsigned mine = 0;
  int const x0 = cell_of(pos.x - M.cs, M.lo.x, M.cs, M.g0), x1 = cell_of(pos.x + M.cs, M.lo.x, M.cs, M.g0);
  int const y0 = cell_of(pos.y - M.cs, M.lo.y, M.cs, M.g1), y1 = cell_of(pos.y + M.cs, M.lo.y, M.cs, M.g1);
  int const z0 = cell_of(pos.z - M.cs, M.lo.z, M.cs, M.g2), z1 = cell_of(pos.z + M.cs, M.lo.z, M.cs, M.g2);
  for (int z = z0; z <= z1; ++z)
    for (int y = y0; y <= y1; ++y) {
      int const row = (z * M.g1 + y) * M.g0;
      int const b = __ldg(&M.start[row + x0]), e = __ldg(&M.start[row + x1 + 1]);
      for (int q0 = b; q0 < e; q0 += 32) {
        int const q = q0 + lane;
        int k = -1;
        if (q < e) {
          float4 const p4 = __ldg(&M.pos[q]);
          f3 const d = mk3(p4.x - pos.x, p4.y - pos.y, p4.z - pos.z);
          if (dot3(d, d) < M.r2) {
            f3 const dir = xyz3(__ldg(&M.dir[q]));
            bool above;
            int const kk = importon_bin(dir, sn, tan, bin, &above);
            f3 const vp = add3(d, scl3(dir, dot3(d, sn)));
            if (above && dot3(vp, vp) < M.r2) k = kk;
          }
        }
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          unsigned const m = __ballot_sync(0xffffffffu, k == t);
          if (lane == t) mine += __popc(m);
        }
      }
    }
  // inclusive prefix sum over lanes 0..15 of (16 + count)
  unsigned acc = lane < 16 ? 16u + mine : 0u;
#pragma unroll
  for (int off = 1; off < 16; off <<= 1) {
    unsigned const o = __shfl_up_sync(0xffffffffu, acc, off);
    if (lane >= off) acc += o;
  }
  return static_cast<float>(acc);
}

// Histograms of an extension queue's hit points (computed as the shading
// kernel computes them) for the importance-driven shading kernel: one warp
// per queue entry.
__global__ void k_importon_query(DevScene S, ImpGrid M, const float4 *qo, const float4 *qd, const float4 *hits,
                                 const int32_t *count, float *cdf) {
  int const n = *count;
  int const lane = threadIdx.x & 31;
  int64_t const warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    float4 const h = hits[i];
    int32_t const code = __float_as_int(h.w);
    if (code < 0) continue;  // the same for the whole warp
    float4 const o4 = qo[i], d4 = qd[i];
    f3 const d = xyz3(d4);
    f3 gn, sn, tan, bin;
    shading_frame(S, code >> 1, code & 1, h.y, h.z, &gn, &sn, &tan, &bin);
    f3 const pos = add3(xyz3(o4), scl3(d, h.x));
    float const c = importon_histogram_warp(M, pos, sn, tan, bin, lane);
    if (lane < 16) cdf[16 * i + lane] = c;
  }
}

// Histograms of caller-given frames (12 floats: position, tangent, binormal,
// shading normal), for tests.
__global__ void k_importon_query_frames(ImpGrid M, const float *fr, int n, float *out) {
  int const lane = threadIdx.x & 31;
  int64_t const warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const float *q = fr + 12 * i;
    float const c = importon_histogram_warp(M, mk3(q[0], q[1], q[2]), mk3(q[9], q[10], q[11]),
                                            mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]), lane);
    if (lane < 16) out[16 * i + lane] = c;
  }
}

ImpGrid grid_view(const ImportonImpl &m) {
  ImpGrid g;
  g.pos = m.d_pos;
  g.dir = m.d_dir;
  g.start = m.d_start;
  g.lo = m.lo;
  g.cs = m.cs;
  g.r2 = m.cfg.radius * m.cfg.radius;
  g.g0 = m.g[0];
  g.g1 = m.g[1];
  g.g2 = m.g[2];
  return g;
}

template <class T>
struct DevArray {
  T *p = nullptr;
  ~DevArray() { cudaFree(p); }
  int alloc(size_t n) {
    cudaError_t const e = cudaMalloc(reinterpret_cast<void **>(&p), std::max<size_t>(n, 1) * sizeof(T));
    return e == cudaSuccess ? XYZGPU_OK
                            : set_error(XYZGPU_E_NOMEM, "importons: allocating %zu bytes failed", n * sizeof(T));
  }
};

// Sorts importons (unsorted device arrays of n) into the map's grid.
int build_grid(ImportonImpl &m, const float4 *pos, const float4 *dir, int64_t n, cudaStream_t st) {
  // grid over the scene box, cells of at least the radius, at most 2^24 cells
  DevScene const &S = m.scene->dev;
  float const r = m.cfg.radius;
  float const ext[3] = {S.bmax.x - S.bmin.x, S.bmax.y - S.bmin.y, S.bmax.z - S.bmin.z};
  float cs = r;
  for (;;) {
    int64_t cells = 1;
    for (int k = 0; k < 3; ++k) cells *= static_cast<int64_t>(ext[k] / cs) + 1;
    if (cells <= (int64_t{1} << 24)) break;
    cs *= 1.25f;
  }
  m.cs = cs;
  m.lo = make_float3(S.bmin.x, S.bmin.y, S.bmin.z);
  for (int k = 0; k < 3; ++k) m.g[k] = static_cast<int>(ext[k] / cs) + 1;
  int64_t const cells = static_cast<int64_t>(m.g[0]) * m.g[1] * m.g[2];
  DevArray<int32_t> key, cnt, fill;
  int rc;
  if ((rc = key.alloc(n)) || (rc = cnt.alloc(cells + 1)) || (rc = fill.alloc(cells + 1))) return rc;
  cudaFree(m.d_start);
  cudaFree(m.d_pos);
  cudaFree(m.d_dir);
  m.d_start = nullptr;
  m.d_pos = m.d_dir = nullptr;
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&m.d_start), (cells + 1) * sizeof(int32_t)));
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&m.d_pos), std::max<int64_t>(n, 1) * sizeof(float4)));
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&m.d_dir), std::max<int64_t>(n, 1) * sizeof(float4)));
  XYZ_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (cells + 1) * sizeof(int32_t), st));
  if (n > 0)
    k_imp_count<<<grid1(m.device, n), kImpThreads, 0, st>>>(pos, n, m.lo, cs, m.g[0], m.g[1], m.g[2], key.p, cnt.p);
  XYZ_CUDA_TRY(cudaGetLastError());
  size_t tmp_bytes = 0;
  XYZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.p, m.d_start, static_cast<int>(cells + 1), st));
  DevArray<uint8_t> tmp;
  if ((rc = tmp.alloc(tmp_bytes))) return rc;
  XYZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, cnt.p, m.d_start, static_cast<int>(cells + 1), st));
  XYZ_CUDA_TRY(cudaMemcpyAsync(fill.p, m.d_start, (cells + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  if (n > 0)
    k_imp_scatter<<<grid1(m.device, n), kImpThreads, 0, st>>>(pos, dir, n, key.p, fill.p, m.d_pos, m.d_dir);
  XYZ_CUDA_TRY(cudaGetLastError());
  XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  m.n = n;
  return XYZGPU_OK;
}

// Traces the light particles and returns the unsorted importons.
int emit(ImportonImpl &m, cudaStream_t st) {
  SceneImpl &s = *m.scene;
  DevScene const &S = s.dev;
  int const P = m.cfg.particles;
  int const depth = m.cfg.max_depth;
  int64_t const cap = static_cast<int64_t>(P) * std::max(1, depth - std::max(0, m.cfg.min_depth));
  DevArray<float4> qo[2], qd[2], hits, ipos, idir;
  DevArray<int32_t> pid[2];
  DevArray<uint32_t> dim[2];
  DevArray<int32_t> counts;  // per depth: queue length, fetch counter
  DevArray<unsigned long long> nimp;
  int rc;
  for (int k = 0; k < 2; ++k)
    if ((rc = qo[k].alloc(P)) || (rc = qd[k].alloc(P)) || (rc = pid[k].alloc(P)) || (rc = dim[k].alloc(P)))
      return rc;
  if ((rc = hits.alloc(P)) || (rc = ipos.alloc(cap)) || (rc = idir.alloc(cap)) ||
      (rc = counts.alloc(2 * (depth + 1))) || (rc = nimp.alloc(1)))
    return rc;
  XYZ_CUDA_TRY(cudaMemsetAsync(counts.p, 0, 2 * (depth + 1) * sizeof(int32_t), st));
  XYZ_CUDA_TRY(cudaMemsetAsync(nimp.p, 0, sizeof(unsigned long long), st));
  if (S.n_lights > 0 && P > 0) {
    int const trace_grid = occupancy_grid(k_particles_trace, m.device);
    ParticleQueue q[2];
    for (int k = 0; k < 2; ++k) q[k] = ParticleQueue{qo[k].p, qd[k].p, pid[k].p, dim[k].p};
    k_particles_start<<<grid1(m.device, P), kImpThreads, 0, st>>>(S, P, m.cfg.seed, q[0], counts.p);
    for (int b = 0; b < depth; ++b) {
      int const cur = b & 1;
      k_particles_trace<<<trace_grid, kThreads, 0, st>>>(S, q[cur].o, q[cur].d, hits.p, counts.p + 2 * b,
                                                          counts.p + 2 * b + 1);
      k_particles_bounce<<<grid1(m.device, P), kImpThreads, 0, st>>>(
          S, b, m.cfg.min_depth, m.cfg.seed, q[cur], hits.p, counts.p + 2 * b, q[cur ^ 1], counts.p + 2 * (b + 1),
          ipos.p, idir.p, nimp.p, cap);
    }
    XYZ_CUDA_TRY(cudaGetLastError());
  }
  unsigned long long n = 0;
  XYZ_CUDA_TRY(cudaMemcpyAsync(&n, nimp.p, sizeof(n), cudaMemcpyDeviceToHost, st));
  XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  if (static_cast<int64_t>(n) > cap) return set_error(XYZGPU_E_LIMIT, "importons: more importons than room for");
  return build_grid(m, ipos.p, idir.p, static_cast<int64_t>(n), st);
}

}  // namespace

int importon_wave_prepare(ImportonImpl &m, int64_t capacity, float **cdf) {
  if (m.cdf_cap < capacity) {
    cudaFree(m.d_cdf);
    m.d_cdf = nullptr;
    m.cdf_cap = 0;
    cudaError_t const e = cudaMalloc(reinterpret_cast<void **>(&m.d_cdf), capacity * 16 * sizeof(float));
    if (e != cudaSuccess)
      return set_error(XYZGPU_E_NOMEM, "render_importon: histogram buffer of %lld entries: %s",
                       static_cast<long long>(capacity), cudaGetErrorString(e));
    m.cdf_cap = capacity;
  }
  *cdf = m.d_cdf;
  return XYZGPU_OK;
}

int importon_query_launch(ImportonImpl &m, const float4 *qo, const float4 *qd, const float4 *hits,
                          const int32_t *count, const DevScene &S, float *cdf, cudaStream_t st) {
  int const grid = occupancy_grid(k_importon_query, m.device);
  k_importon_query<<<grid, kThreads, 0, st>>>(S, grid_view(m), qo, qd, hits, count, cdf);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int importon_guide_bounces(const ImportonImpl &m) { return m.cfg.guide_bounces; }

}  // namespace xyzgpu

using namespace xyzgpu;

struct xyzgpu_importons_s {
  ImportonImpl m;
};

extern "C" {

void xyzgpu_importon_config_default(xyzgpu_importon_config *c) {
  if (!c) return;
  c->particles = 100000;  // CONFIG_EMITED_SIZE (xyz/core/config.hpp:57)
  c->max_depth = 16;      // XYZ_CONFIG_kMaxRandomWalkDepth (config.hpp:30)
  c->min_depth = 1;
  c->radius = 0.1f;       // CONFIG_SEARCH_RADIUS (config.hpp:56)
  c->seed = 0;
  c->guide_bounces = 1 << 20;
}

void xyzgpu_importons_destroy(xyzgpu_importons h) {
  if (!h) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->m.device);
  cudaDeviceSynchronize();
  cudaFree(h->m.d_pos);
  cudaFree(h->m.d_dir);
  cudaFree(h->m.d_start);
  cudaFree(h->m.d_cdf);
  cudaSetDevice(prev);
  delete h;
}

int xyzgpu_importons_create(xyzgpu_scene scene, const xyzgpu_importon_config *cfg, const float *importons,
                            int64_t n_importons, void *stream, xyzgpu_importons *out) {
  clear_error();
  if (!scene || !out || (n_importons > 0 && !importons) || n_importons < 0)
    return set_error(XYZGPU_E_INVALID, "importons_create: bad argument");
  *out = nullptr;
  xyzgpu_importon_config c;
  if (cfg)
    c = *cfg;
  else
    xyzgpu_importon_config_default(&c);
  if (c.particles < 0 || c.max_depth < 1 || c.max_depth > 1000 || c.min_depth < 0 || !(c.radius > 0.0f) ||
      !std::isfinite(c.radius) || c.guide_bounces < 0)
    return set_error(XYZGPU_E_INVALID, "importons_create: configuration out of range");
  auto *h = new (std::nothrow) xyzgpu_importons_s();
  if (!h) return set_error(XYZGPU_E_NOMEM, "importons_create: host allocation failed");
  ImportonImpl &m = h->m;
  m.scene = reinterpret_cast<SceneImpl *>(scene);
  if (m.scene->n_specular) {
    delete h;
    return set_error(XYZGPU_E_INVALID, "importons_create: scenes with mirror or metal materials are not supported");
  }
  m.device = m.scene->device;
  m.cfg = c;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  int rc = XYZGPU_OK;
  if (cudaSetDevice(m.device) != cudaSuccess) rc = set_error(XYZGPU_E_CUDA, "importons_create: cudaSetDevice failed");
  if (!rc && importons) {
    // a given map: (position, incoming direction) per importon
    std::vector<float4> p(static_cast<size_t>(n_importons)), d(static_cast<size_t>(n_importons));
    for (int64_t i = 0; i < n_importons; ++i) {
      const float *q = importons + 6 * i;
      p[i] = make_float4(q[0], q[1], q[2], 0.0f);
      d[i] = make_float4(q[3], q[4], q[5], 0.0f);
    }
    DevArray<float4> dp, dd;
    if (!(rc = dp.alloc(n_importons)) && !(rc = dd.alloc(n_importons))) {
      if (cudaMemcpy(dp.p, p.data(), n_importons * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dd.p, d.data(), n_importons * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error(XYZGPU_E_CUDA, "importons_create: upload failed");
      else
        rc = build_grid(m, dp.p, dd.p, n_importons, st);
    }
  } else if (!rc) {
    rc = emit(m, st);
  }
  if (rc) {
    xyzgpu_importons_destroy(h);
    return rc;
  }
  *out = h;
  return XYZGPU_OK;
}

int xyzgpu_importons_get(xyzgpu_importons h, float *importons, int64_t *n) {
  clear_error();
  if (!h || !n) return set_error(XYZGPU_E_INVALID, "importons_get: bad argument");
  *n = h->m.n;
  if (!importons || h->m.n == 0) return XYZGPU_OK;
  XYZ_CUDA_TRY(cudaSetDevice(h->m.device));
  std::vector<float4> p(static_cast<size_t>(h->m.n)), d(static_cast<size_t>(h->m.n));
  XYZ_CUDA_TRY(cudaMemcpy(p.data(), h->m.d_pos, h->m.n * sizeof(float4), cudaMemcpyDeviceToHost));
  XYZ_CUDA_TRY(cudaMemcpy(d.data(), h->m.d_dir, h->m.n * sizeof(float4), cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < h->m.n; ++i) {
    float *q = importons + 6 * i;
    q[0] = p[i].x, q[1] = p[i].y, q[2] = p[i].z, q[3] = d[i].x, q[4] = d[i].y, q[5] = d[i].z;
  }
  return XYZGPU_OK;
}

int xyzgpu_importons_query(xyzgpu_importons h, const float *frames, int n, float *hist, void *stream) {
  clear_error();
  if (!h || n < 0 || (n > 0 && (!frames || !hist))) return set_error(XYZGPU_E_INVALID, "importons_query: bad argument");
  if (n == 0) return XYZGPU_OK;
  XYZ_CUDA_TRY(cudaSetDevice(h->m.device));
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  k_importon_query_frames<<<grid1(h->m.device, n), kImpThreads, 0, st>>>(grid_view(h->m), frames, n, hist);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int xyzgpu_render_importon(xyzgpu_importons h, const xyzgpu_camera *cam, const xyzgpu_render_params *rp,
                           float *film, void *stream) {
  clear_error();
  if (!h || !cam || !rp || !film) return set_error(XYZGPU_E_INVALID, "render_importon: null argument");
  if (rp->spectral != XYZGPU_SPECTRAL_OFF || rp->profile == XYZGPU_PROFILE_COUNTERS)
    return set_error(XYZGPU_E_INVALID, "render_importon: the XYZ film mode only, profile off or timing");
  int const rc = check_render_args("render_importon", reinterpret_cast<xyzgpu_scene>(h->m.scene), cam, rp);
  if (rc) return rc;
  XYZ_CUDA_TRY(cudaSetDevice(h->m.device));
  ImportonHooks hooks{&h->m};
  return render_launch(*h->m.scene, *cam, *rp, film, static_cast<cudaStream_t>(stream), nullptr, nullptr, &hooks);
}

}  // extern "C"
