// Closest-hit entry point (xyzgpu_trace_closest): the batch form of
// Scene::FindIntersection (xyz/core/scene.hpp:277-295).
//
// Persistent warps with per-lane refill (trace_persistent in traverse.cuh):
// rays are taken from a global counter as lanes free up, so long and short
// rays balance across lanes and SMs.  Rays are read as two 16-byte vectors and
// hits written as one.
#include "scene.h"
#include "traverse.cuh"

namespace xyzgpu {
namespace {

constexpr int kTraceThreads = 128;

// Rays as 8 floats (o, tmin, d, tmax); hits as (t, f, g, id << 1 | back).
struct ApiSink {
  const float4 *__restrict__ rays;
  float4 *__restrict__ hits;
  uint32_t n_rays, n_hits;
  XYZ_DEV void load(int i, f3 &o, f3 &d, float &tmin, float &tmax) const {
    float4 const a = __ldg(&rays[2 * i + 0]);
    float4 const b = __ldg(&rays[2 * i + 1]);
    o = xyz3(a);
    d = xyz3(b);
    tmin = a.w;
    tmax = b.w;
  }
  XYZ_DEV void store(int i, const RayHit &h) {
    int32_t const code = h.id >= 0 ? ((h.id << 1) | h.back) : -1;
    hits[i] = make_float4(h.id >= 0 ? h.t : 0.0f, h.f, h.g, __int_as_float(code));
    ++n_rays;
    n_hits += h.id >= 0;
  }
};

template <bool kCount>
__global__ void __launch_bounds__(kTraceThreads)
    k_trace_api(DevScene S, const float4 *__restrict__ rays, int n, float4 *__restrict__ hits,
                int *__restrict__ fetch, unsigned long long *__restrict__ counts) {
  int const lane = threadIdx.x & 31;
  TraceCount c{0u, 0u, 0u};
  ApiSink sink{rays, hits, 0u, 0u};
  trace_persistent<kCount>(S, n, fetch, sink, c);
  uint32_t const n_rays = sink.n_rays, n_hits = sink.n_hits;
  if (kCount) {
    unsigned long long v[5] = {n_rays, c.nodes, c.leaves, c.tris, n_hits};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      unsigned long long x = v[k];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
      if (lane == 0) atomicAdd(&counts[k], x);
    }
  }
}

template <bool kCount>
int grid_for(int device) {
  static int blocks = 0;
  if (blocks == 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_api<kCount>, kTraceThreads,
                                                      0) != cudaSuccess ||
        per_sm <= 0)
      per_sm = 4;
    blocks = per_sm * sm_count(device);
  }
  return blocks;
}

}  // namespace

int trace_api_launch(SceneImpl &s, const float *rays, int n, float *hits, cudaStream_t st,
                     xyzgpu_trace_counters *counters) {
  if (counters) *counters = xyzgpu_trace_counters{0, 0, 0, 0, 0};
  if (n == 0) return XYZGPU_OK;
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  XYZ_CUDA_TRY(cudaMemsetAsync(s.d_fetch, 0, sizeof(int32_t), st));
  const float4 *r4 = reinterpret_cast<const float4 *>(rays);
  float4 *h4 = reinterpret_cast<float4 *>(hits);
  if (counters) {
    XYZ_CUDA_TRY(cudaMemsetAsync(s.d_trace_counts, 0, 8 * sizeof(unsigned long long), st));
    k_trace_api<true><<<grid_for<true>(s.device), kTraceThreads, 0, st>>>(s.dev, r4, n, h4, s.d_fetch,
                                                                        s.d_trace_counts);
    XYZ_CUDA_TRY(cudaGetLastError());
    unsigned long long c[8];
    XYZ_CUDA_TRY(cudaMemcpyAsync(c, s.d_trace_counts, sizeof(c), cudaMemcpyDeviceToHost, st));
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    counters->rays = c[0];
    counters->nodes_visited = c[1];
    counters->leaves_visited = c[2];
    counters->tri_tests = c[3];
    counters->hits = c[4];
  } else {
    k_trace_api<false><<<grid_for<false>(s.device), kTraceThreads, 0, st>>>(s.dev, r4, n, h4, s.d_fetch,
                                                                          nullptr);
    XYZ_CUDA_TRY(cudaGetLastError());
  }
  return XYZGPU_OK;
}

}  // namespace xyzgpu
