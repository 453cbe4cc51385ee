// Host side of xyzgpu_render / xyzgpu_adjoint (single scene) and
// xyzgpu_render_noalloc; the kernels are in wavefront.cuh.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <mutex>

#include "wavefront.cuh"

namespace xyzgpu {
namespace {
constexpr int64_t kMaxDefaultWave = int64_t{1} << 26;
constexpr int64_t kMaxGuidedWave = int64_t{1} << 23;

// Grids of one full wave of resident CTAs per kernel variant on a device (the
// grid-stride loops give every CTA an equal share, so a grid larger than what
// fits at once would run a second, tail wave).  Sized once per device and
// published under a mutex only when complete, so threads rendering on several
// devices never see a partly filled entry or another device's grids.
struct Grids {
  int raygen, trace_e, trace_s, trace_s_adj, trace_s_guide, trace_s_imp;
  int shade, shade_adj, shade_guide, shade_sp, shade_imp, film;
};

Grids wave_grids(int device) {
  static std::mutex mu;
  static Grids table[64];
  static bool ready[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  int const d = device & 63;
  if (!ready[d]) {
    Grids g;
    g.raygen = occupancy_grid(k_raygen<false>, device);
    g.trace_e = occupancy_grid(k_trace_queue<false, false>, device);
    g.trace_s = occupancy_grid(k_trace_queue<true, false>, device);
    g.trace_s_adj = occupancy_grid(k_trace_queue<true, false, kModeAdjoint>, device);
    g.trace_s_guide = occupancy_grid(k_trace_queue<true, false, kModeGuided>, device);
    g.shade = occupancy_grid(k_shade<kModePlain>, device);
    g.shade_adj = occupancy_grid(k_shade<kModeAdjoint>, device);
    g.shade_guide = occupancy_grid(k_shade<kModeGuided>, device);
    g.shade_sp = occupancy_grid(k_shade_spectral, device);
    g.trace_s_imp = occupancy_grid(k_trace_queue<true, false, kModeImporton>, device);
    g.shade_imp = occupancy_grid(k_shade<kModeImporton>, device);
    g.film = occupancy_grid(k_film, device);
    table[d] = g;
    ready[d] = true;
  }
  return table[d];
}
}  // namespace

extern const int64_t kBytesPerPath = 3 * sizeof(float4) + sizeof(uint32_t) +  // beta, radiance, hits, misc
                                  2 * (2 * sizeof(float4) + sizeof(int32_t)) +  // extension queues
                                  4 * sizeof(float4) + sizeof(int32_t) +         // shadow queue
                                  sizeof(float) + sizeof(int32_t);               // spectral fsn, slot

SharedWaves &shared_waves(int device) {
  static SharedWaves pool[64];
  return pool[device & 63];
}

void free_wave_buffers(RenderWorkspace &w) {
  cudaFree(w.beta);
  cudaFree(w.misc);
  cudaFree(w.radiance);
  for (int q = 0; q < 2; ++q) {
    cudaFree(w.q_o[q]);
    cudaFree(w.q_d[q]);
    cudaFree(w.q_slot[q]);
  }
  cudaFree(w.hits);
  cudaFree(w.s_o);
  cudaFree(w.s_d);
  cudaFree(w.s_pb);
  cudaFree(w.s_m);
  cudaFree(w.s_target);
  cudaFree(w.fsn);
  cudaFree(w.s_slot);
  cudaFree(w.counts);
  w.fsn = nullptr;
  w.s_slot = nullptr;
  w.beta = w.radiance = w.hits = w.s_o = w.s_d = w.s_pb = w.s_m = nullptr;
  w.misc = nullptr;
  w.q_o[0] = w.q_o[1] = w.q_d[0] = w.q_d[1] = nullptr;
  w.q_slot[0] = w.q_slot[1] = w.s_target = w.counts = nullptr;
  w.capacity = 0;
  w.max_iters = 0;
}

int ensure_wave_buffers(RenderWorkspace &w, int64_t capacity, int iters) {
  if (w.capacity >= capacity && w.max_iters >= iters) return XYZGPU_OK;
  capacity = std::max(capacity, w.capacity);
  iters = std::max(iters, w.max_iters);
  free_wave_buffers(w);
  size_t const c = static_cast<size_t>(capacity);
#define XYZ_ALLOC(ptr, bytes)                                                         \
  do {                                                                                \
    cudaError_t const e_ = cudaMalloc(reinterpret_cast<void **>(&(ptr)), (bytes));    \
    if (e_ != cudaSuccess) {                                                          \
      free_wave_buffers(w);                                                           \
      return set_error(e_ == cudaErrorMemoryAllocation ? XYZGPU_E_NOMEM : XYZGPU_E_CUDA, \
                       "render: allocating %zu bytes of wave buffers failed: %s",     \
                       static_cast<size_t>(bytes), cudaGetErrorString(e_));           \
    }                                                                                 \
  } while (0)
  XYZ_ALLOC(w.beta, c * sizeof(float4));
  XYZ_ALLOC(w.misc, c * sizeof(uint32_t));
  XYZ_ALLOC(w.radiance, c * sizeof(float4));
  for (int q = 0; q < 2; ++q) {
    XYZ_ALLOC(w.q_o[q], c * sizeof(float4));
    XYZ_ALLOC(w.q_d[q], c * sizeof(float4));
    XYZ_ALLOC(w.q_slot[q], c * sizeof(int32_t));
  }
  XYZ_ALLOC(w.hits, c * sizeof(float4));
  XYZ_ALLOC(w.s_o, c * sizeof(float4));
  XYZ_ALLOC(w.s_d, c * sizeof(float4));
  XYZ_ALLOC(w.s_pb, c * sizeof(float4));
  XYZ_ALLOC(w.s_m, c * sizeof(float4));
  XYZ_ALLOC(w.s_target, c * sizeof(int32_t));
  XYZ_ALLOC(w.fsn, c * sizeof(float));
  XYZ_ALLOC(w.s_slot, c * sizeof(int32_t));
  XYZ_ALLOC(w.counts, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t));
#undef XYZ_ALLOC
  w.capacity = capacity;
  w.max_iters = iters;
  return XYZGPU_OK;
}


// Frees a scene's own render state (profiling tally and events, host-film
// staging); the wave buffers belong to the device.
void render_workspace_free(RenderWorkspace &w) {
  cudaFree(w.tally);
  for (cudaEvent_t e : w.events) cudaEventDestroy(e);
  cudaFree(w.film_dev);
  cudaFreeHost(w.film_pinned);
  w = RenderWorkspace{};
}

int render_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp, float *film,
                  cudaStream_t st, const AdjointArgs *adj, const GuideHooks *guide, const ImportonHooks *imp) {
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  // a band of rows (every row_step-th row of it) renders the same pixels and
  // paths as the full image
  int64_t const row0 = rp.row_end > 0 ? rp.row_begin : 0;
  int64_t const row_step = rp.row_end > 0 && rp.row_step > 1 ? rp.row_step : 1;
  int64_t const rows = rp.row_end > 0 ? (rp.row_end - rp.row_begin + row_step - 1) / row_step : rp.height;
  int64_t const npix_total = static_cast<int64_t>(rp.width) * rows;
  int64_t const film_elems = 3 * static_cast<int64_t>(rp.width) * rp.height;
  int const iters = rp.max_depth;

  CamDev const C = camera_setup(cam, rp.width, rp.height);

  float *film_dev = film;
  RenderWorkspace &w = s.ws;
  if (!w.tally) XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&w.tally), kTallyWords * sizeof(unsigned long long)));
  SharedWaves &sw = shared_waves(s.device);
  std::lock_guard<std::mutex> lock(sw.mu);
  // Wave size: the caller's, else every path of the call (at most 2^26),
  // bounded by half of the free device memory.
  int64_t cap = rp.wave_paths;
  if (cap <= 0) {
    cap = std::min<int64_t>(kMaxDefaultWave, std::max<int64_t>(1, npix_total * rp.spp));
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      int64_t const afford = static_cast<int64_t>((free_b / 2 + sw.ws.capacity * kBytesPerPath) / kBytesPerPath);
      cap = std::min(cap, std::max<int64_t>(afford, int64_t{1} << 20));
    }
    cap = std::max(cap, sw.ws.capacity);
    // guided waves also hold a mixture (80 B) and training records per path,
    // importance-driven waves a histogram (64 B) per path
    if (guide || imp) cap = std::min<int64_t>(cap, kMaxGuidedWave);
  }
  if (sw.done && sw.last != st) XYZ_CUDA_TRY(cudaStreamWaitEvent(st, sw.done, 0));
  int rc = ensure_wave_buffers(sw.ws, cap, iters);
  if (rc) return rc;
  if (!sw.done) XYZ_CUDA_TRY(cudaEventCreateWithFlags(&sw.done, cudaEventDisableTiming));
  RenderWorkspace const &wv = sw.ws;
  // Host films go through one device film and one pinned buffer per device
  // (kept across scenes, so a program that creates a scene per frame does not
  // pin and unpin host memory every time); the device lock held for the whole
  // call serialises their use, and the call returns only after the read-back.
  RenderWorkspace &fs = sw.ws;
  // A host film in page-locked memory is copied to and from directly.
  bool film_locked = false;
  if (!adj && rp.film_location == XYZGPU_FILM_HOST) {
    cudaPointerAttributes pa;
    film_locked = cudaPointerGetAttributes(&pa, film) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
  }
  if (!adj && rp.film_location == XYZGPU_FILM_HOST) {
    if (fs.film_elems < film_elems) {
      XYZ_CUDA_TRY(cudaStreamSynchronize(st));
      cudaFree(fs.film_dev);
      cudaFreeHost(fs.film_pinned);
      fs.film_dev = nullptr;
      fs.film_pinned = nullptr;
      fs.film_elems = 0;
      XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&fs.film_dev), film_elems * sizeof(float)));
      XYZ_CUDA_TRY(cudaMallocHost(reinterpret_cast<void **>(&fs.film_pinned), film_elems * sizeof(float)));
      fs.film_elems = film_elems;
    }
    film_dev = fs.film_dev;
    if (rp.accumulate && film_locked) {
      XYZ_CUDA_TRY(cudaMemcpyAsync(film_dev, film, film_elems * sizeof(float), cudaMemcpyHostToDevice, st));
    } else if (rp.accumulate) {
      std::memcpy(fs.film_pinned, film, film_elems * sizeof(float));
      XYZ_CUDA_TRY(cudaMemcpyAsync(film_dev, fs.film_pinned, film_elems * sizeof(float),
                                   cudaMemcpyHostToDevice, st));
    }
  }
  if (!adj && !rp.accumulate) XYZ_CUDA_TRY(cudaMemsetAsync(film_dev, 0, film_elems * sizeof(float), st));
  float4 *ltot = nullptr;
  if (adj) {
    cudaError_t const e = cudaMallocAsync(reinterpret_cast<void **>(&ltot), static_cast<size_t>(cap) * sizeof(float4), st);
    if (e != cudaSuccess)
      return set_error(e == cudaErrorMemoryAllocation ? XYZGPU_E_NOMEM : XYZGPU_E_CUDA,
                       "adjoint: allocating the primal radiance of %lld paths failed: %s",
                       static_cast<long long>(cap), cudaGetErrorString(e));
  }
  // Adjoint: the primal pass records each path's extension hits and shadow
  // results per bounce (20 B per path and bounce) so that the replay traces no
  // rays; without room for them the replay traces its paths again.
  float4 *hit_cache = nullptr;
  float *vis_cache = nullptr;
  // XYZGPU_ADJOINT_TRACE_REPLAY set: the replay traces (no recorded intersections)
  if (adj && !std::getenv("XYZGPU_ADJOINT_TRACE_REPLAY")) {
    int64_t const per_wave = std::min<int64_t>(cap, std::max<int64_t>(1, npix_total * rp.spp));
    size_t const entries = static_cast<size_t>(per_wave) * static_cast<size_t>(iters);
    if (cudaMallocAsync(reinterpret_cast<void **>(&hit_cache), entries * sizeof(float4), st) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void **>(&vis_cache), entries * sizeof(float), st) != cudaSuccess) {
      cudaGetLastError();  // not an error: the replay traces instead
      if (hit_cache) cudaFreeAsync(hit_cache, st);
      if (vis_cache) cudaFreeAsync(vis_cache, st);
      hit_cache = nullptr;
      vis_cache = nullptr;
    }
  }
  // frees the adjoint's buffers on every return below
  struct FreeAsync {
    void *p;
    cudaStream_t st;
    ~FreeAsync() {
      if (p) cudaFreeAsync(p, st);
    }
  } ltot_guard{ltot, st}, hit_guard{hit_cache, st}, vis_guard{vis_cache, st};

  Grids const G = wave_grids(s.device);
  int const prof = rp.profile;
  bool const spectral = rp.spectral != XYZGPU_SPECTRAL_OFF;
  bool const timing = prof == XYZGPU_PROFILE_TIMING;
  bool const counting = prof == XYZGPU_PROFILE_COUNTERS;
  XYZ_CUDA_TRY(cudaMemsetAsync(w.tally, 0, kTallyWords * sizeof(unsigned long long), st));
  w.profile_iters = iters;
  s.event_class.clear();
  size_t n_ev = 0;
  // Records the start or end event of a launch of `cls` (TIMING renders).
  auto mark = [&](int cls, bool start) -> int {
    if (!timing) return XYZGPU_OK;
    if (n_ev == w.events.size()) {
      cudaEvent_t e;
      XYZ_CUDA_TRY(cudaEventCreate(&e));
      w.events.push_back(e);
    }
    XYZ_CUDA_TRY(cudaEventRecord(w.events[n_ev++], st));
    if (start) s.event_class.push_back(cls);
    return XYZGPU_OK;
  };
  unsigned long long *const pc = w.tally + 8;

  WaveArgs A;
  std::memset(&A, 0, sizeof(A));
  A.S = s.dev;
  A.cam = C;
  A.W = rp.width;
  A.H = rp.height;
  A.kmax = rp.max_depth + 1;
  A.rr_start = rp.rr_start_depth;
  A.rr_threshold = rp.rr_threshold;
  A.seed = rp.seed;
  A.beta = wv.beta;
  A.misc = wv.misc;
  A.radiance = wv.radiance;
  for (int q = 0; q < 2; ++q) {
    A.q_o[q] = wv.q_o[q];
    A.q_d[q] = wv.q_d[q];
    A.q_slot[q] = wv.q_slot[q];
  }
  A.hits = wv.hits;
  A.s_o = wv.s_o;
  A.s_d = wv.s_d;
  A.s_pb = wv.s_pb;
  A.s_m = wv.s_m;
  A.s_target = wv.s_target;
  A.counts = wv.counts;
  A.spectral = rp.spectral;
  A.hero = spectral ? rp.hero_wavelengths : 1;
  A.wl_dim = cam.pinhole ? 4u : 6u;
  A.fsn = wv.fsn;
  A.s_slot = wv.s_slot;
  if (adj) {
    A.ltot = ltot;
    A.dfilm = adj->d_film;
    A.g_alb = adj->g_albedo;
    A.g_em = adj->g_emission;
  }
  GuideWave gw;
  if (guide) {
    // a wave never holds more paths than the call renders
    int64_t const need = std::min<int64_t>(cap, std::max<int64_t>(1, npix_total * rp.spp));
    int const r = guide_wave_prepare(*guide->g, need, guide->train, st, &gw);
    if (r) return r;
    A.mix = static_cast<const __half *>(gw.mix);
    A.guide_alpha = gw.alpha;
    A.records = gw.records;
    A.train_bounces = gw.train_bounces;
  }

  float *imp_cdf = nullptr;
  int imp_bounces = 0;
  if (imp) {
    int64_t const need = std::min<int64_t>(cap, std::max<int64_t>(1, npix_total * rp.spp));
    int const r = importon_wave_prepare(*imp->m, need, &imp_cdf);
    if (r) return r;
    imp_bounces = importon_guide_bounces(*imp->m);
  }

  xyzgpu_render_counters rc_out{};
  uint64_t launches = 0;
  // Wave shape: whole samples of as many pixels as fit, else pixel blocks.
  int64_t const spp_per_wave = std::max<int64_t>(1, std::min<int64_t>(rp.spp, cap / std::max<int64_t>(1, npix_total)));
  int64_t const pix_per_wave = std::min<int64_t>(npix_total, cap);
  for (int64_t s0 = 0; s0 < rp.spp; s0 += spp_per_wave) {
    int const ns = static_cast<int>(std::min<int64_t>(spp_per_wave, rp.spp - s0));
    for (int64_t p0 = 0; p0 < npix_total; p0 += pix_per_wave) {
      A.p0 = p0;
      A.row0 = row0;
      A.row_step = static_cast<int>(row_step);
      A.npix = std::min<int64_t>(pix_per_wave, npix_total - p0);
      A.s0 = static_cast<uint32_t>(rp.spp_offset + s0);
      A.nsamp = ns;
      A.npaths = A.npix * ns;
      XYZ_CUDA_TRY(cudaMemsetAsync(wv.counts, 0, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t), st));
      if (A.train_bounces > 0)
        XYZ_CUDA_TRY(cudaMemsetAsync(A.records, 0, static_cast<size_t>(A.npaths) * A.train_bounces * 16 * sizeof(float), st));
      bool const cached = hit_cache != nullptr;
      if (cached) {
        // all-ones words are NaN: "no visible shadow ray" until the primal writes one
        XYZ_CUDA_TRY(cudaMemsetAsync(vis_cache, 0xff, static_cast<size_t>(A.npaths) * iters * sizeof(float), st));
        A.hit_cache = hit_cache;
        A.vis_cache = vis_cache;
        A.cache_stride = iters;
      }
      int const gr = static_cast<int>(std::min<int64_t>(G.raygen, (A.npaths + kThreads - 1) / kThreads));
#define XYZ_MARK(cls, start)              \
  do {                                    \
    int const m_ = mark((cls), (start));  \
    if (m_) return m_;                    \
  } while (0)
      // One pass over the wave: camera rays, then per bounce closest hit,
      // shading and shadow rays.  The adjoint runs it twice (primal, replay).
      auto pass = [&](bool replay) -> int {
        XYZ_MARK(0, true);
        k_raygen<false><<<gr, kThreads, 0, st>>>(A);
        XYZ_MARK(0, false);
        ++launches;
        // a replay over cached intersections traces no rays
        bool const trace = !(replay && cached);
        for (int b = 0; b < iters; ++b) {
          XYZ_MARK(1, true);
          if (!trace)
            ;
          else if (counting)
            k_trace_queue<false, true><<<G.trace_e, kThreads, 0, st>>>(A, b, pc);
          else
            k_trace_queue<false, false><<<G.trace_e, kThreads, 0, st>>>(A, b, pc);
          XYZ_MARK(1, false);
          // (the last bounce only meets the depth cap: no sampling, no inference;
          // beyond guide_bounces the guided kernels sample Lambert alone)
          bool const guided_here = guide && b < iters - 1 && b < gw.guide_bounces;
          A.guide_alpha = guided_here ? gw.alpha : 0.0f;
          if (guided_here) {
            int const qi = b & 1;
            XYZ_MARK(5, true);
            int const r = guide_infer_launch(*guide->g, A.q_o[qi], A.q_d[qi], A.hits,
                                             A.counts + b * kCountStride + kCExt, A.S, gw.mix, st);
            if (r) return r;
            XYZ_MARK(5, false);
            ++launches;
          }
          // importance-driven: the histograms of this bounce's hit points
          bool const imp_here = imp && b < iters - 1 && b < imp_bounces;
          A.imp_cdf = imp_here ? imp_cdf : nullptr;
          if (imp_here) {
            int const qi = b & 1;
            XYZ_MARK(5, true);
            int const r = importon_query_launch(*imp->m, A.q_o[qi], A.q_d[qi], A.hits,
                                                A.counts + b * kCountStride + kCExt, A.S, imp_cdf, st);
            if (r) return r;
            XYZ_MARK(5, false);
            ++launches;
          }
          XYZ_MARK(2, true);
          if (spectral)
            k_shade_spectral<<<G.shade_sp, kThreads, 0, st>>>(A, b);
          else if (imp)
            k_shade<kModeImporton><<<G.shade_imp, kThreads, 0, st>>>(A, b);
          else if (guide)
            k_shade<kModeGuided><<<G.shade_guide, kThreads, 0, st>>>(A, b);
          else if (replay)
            k_shade<kModeAdjoint><<<G.shade_adj, kThreads, 0, st>>>(A, b);
          else
            k_shade<kModePlain><<<G.shade, kThreads, 0, st>>>(A, b);
          XYZ_MARK(2, false);
          XYZ_MARK(3, true);
          if (!trace)
            ;
          else if (counting)
            k_trace_queue<true, true><<<G.trace_s, kThreads, 0, st>>>(A, b, pc);
          else if (replay)
            k_trace_queue<true, false, kModeAdjoint><<<G.trace_s_adj, kThreads, 0, st>>>(A, b, pc);
          else if (guide)
            k_trace_queue<true, false, kModeGuided><<<G.trace_s_guide, kThreads, 0, st>>>(A, b, pc);
          else if (imp)
            k_trace_queue<true, false, kModeImporton><<<G.trace_s_imp, kThreads, 0, st>>>(A, b, pc);
          else
            k_trace_queue<true, false><<<G.trace_s, kThreads, 0, st>>>(A, b, pc);
          XYZ_MARK(3, false);
          launches += trace ? 3 : 1;
        }
        return XYZGPU_OK;
      };
      int const pr = pass(false);
      if (pr) return pr;
      int const gf = static_cast<int>(std::min<int64_t>(G.film, (A.npix + kThreads - 1) / kThreads));
      if (adj) {
        int const gs = static_cast<int>(std::min<int64_t>(G.film, (A.npaths + kThreads - 1) / kThreads));
        k_adj_stash<<<gs, kThreads, 0, st>>>(A);
        ++launches;
        if (cached) {
          // the counters of an adjoint with cached intersections are the primal's rays
          k_tally<<<1, 32, 0, st>>>(A, iters, w.tally);
          ++launches;
        }
        XYZ_CUDA_TRY(cudaMemsetAsync(wv.counts, 0, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t), st));
        int const rr = pass(true);
        if (rr) return rr;
      } else {
        XYZ_MARK(4, true);
        if (spectral)
          k_film_spectral<<<gf, kThreads, 0, st>>>(A, film_dev);
        else
          k_film<<<gf, kThreads, 0, st>>>(A, film_dev);
        XYZ_MARK(4, false);
        ++launches;
      }
      if (!(adj && cached)) {
        k_tally<<<1, 32, 0, st>>>(A, iters, w.tally);
        ++launches;
      }
      XYZ_CUDA_TRY(cudaGetLastError());
      if (guide && A.train_bounces > 0) {
        XYZ_MARK(5, true);
        int const r = guide_train_on_wave(*guide->g, A.radiance, A.npaths, st);
        if (r) return r;
        XYZ_MARK(5, false);
      }
#undef XYZ_MARK
      rc_out.paths += static_cast<uint64_t>(A.npaths);
      rc_out.waves += 1;
    }
  }
  XYZ_CUDA_TRY(cudaEventRecord(sw.done, st));
  sw.last = st;
  if (!adj && rp.film_location == XYZGPU_FILM_HOST && film_locked) {
    XYZ_CUDA_TRY(cudaMemcpyAsync(film, film_dev, film_elems * sizeof(float), cudaMemcpyDeviceToHost, st));
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  } else if (!adj && rp.film_location == XYZGPU_FILM_HOST) {
    XYZ_CUDA_TRY(cudaMemcpyAsync(fs.film_pinned, film_dev, film_elems * sizeof(float), cudaMemcpyDeviceToHost, st));
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(film, fs.film_pinned, film_elems * sizeof(float));
  }
  rc_out.kernel_launches = launches;
  s.counters = rc_out;
  s.profile_mode = prof;
  s.profile_pending = true;
  return XYZGPU_OK;
}

// Reads back the device tallies (and event times) of the last render.
int render_collect(SceneImpl &s) {
  if (!s.profile_pending) return XYZGPU_OK;
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  RenderWorkspace &w = s.ws;
  XYZ_CUDA_TRY(cudaDeviceSynchronize());
  unsigned long long t[kTallyWords];
  XYZ_CUDA_TRY(cudaMemcpy(t, w.tally, sizeof(t), cudaMemcpyDeviceToHost));
  s.counters.extension_rays = t[0];
  s.counters.shadow_rays = t[1];
  s.counters.shadow_hits_visible = t[2];
  if (s.profile_mode != XYZGPU_PROFILE_OFF) {
    xyzgpu_render_profile &p = s.profile;
    p = xyzgpu_render_profile{};
    p.ext_rays = t[0];
    p.shadow_rays = t[1];
    p.shadow_visible = t[2];
    p.iterations = static_cast<uint32_t>(std::min(w.profile_iters, XYZGPU_PROFILE_MAX_ITERS));
    for (int b = 0; b < XYZGPU_PROFILE_MAX_ITERS; ++b) {
      p.ext_rays_by_iter[b] = t[kTallyIterBase + b];
      p.shadow_rays_by_iter[b] = t[kTallyIterBase + XYZGPU_PROFILE_MAX_ITERS + b];
    }
    if (s.profile_mode == XYZGPU_PROFILE_COUNTERS) {
      p.ext_nodes = t[8];
      p.ext_leaves = t[9];
      p.ext_tri_tests = t[10];
      p.shadow_nodes = t[11];
      p.shadow_leaves = t[12];
      p.shadow_tri_tests = t[13];
    }
    if (s.profile_mode == XYZGPU_PROFILE_TIMING) {
      for (size_t i = 0; i < s.event_class.size(); ++i) {
        float ms = 0.0f;
        XYZ_CUDA_TRY(cudaEventElapsedTime(&ms, w.events[2 * i], w.events[2 * i + 1]));
        int const c = s.event_class[i];
        p.launches[c] += 1;
        p.ms[c] += ms;
      }
    }
  }
  s.profile_pending = false;
  return XYZGPU_OK;
}

// ---------------------------------------------------------------------------
// xyzgpu_render_noalloc: rendering for callers that cannot allocate.
//
// Some hosts must not allocate device memory once they are running: a
// renderer embedded in an application that hands all GPU memory to its own
// pool at start-up, a real-time loop that may not enter the driver's allocator
// (and its implicit synchronisation) in the middle of a frame, or a process
// whose memory budget is fixed when it starts.  xyzgpu_render allocates the
// per-scene path state and queues on its first call and again whenever a
// larger wave is asked for; this entry point instead keeps them in one
// file-scope device array of fixed size, so it performs no allocation at all.
// The scene (created beforehand) and the device film are the caller's.
//
// The array is XYZGPU_NOALLOC_SCRATCH_BYTES on every device that loads the
// library, held until the process exits.  It holds the state of at most
// XYZGPU_NOALLOC_MAX_WAVE_PATHS paths in flight, so large images render in
// more, smaller waves than xyzgpu_render uses (same image, lower throughput).
// Every call on a device shares the array and it keeps the previous call's
// contents: calls that overlap on the GPU (different streams, threads or
// scenes) race and must be serialised by the caller.
namespace {

constexpr int64_t kNoAllocPaths = XYZGPU_NOALLOC_MAX_WAVE_PATHS;
constexpr int kNoAllocDepth = XYZGPU_NOALLOC_MAX_DEPTH;
constexpr size_t kSeg = 256;
constexpr size_t seg(size_t bytes) { return (bytes + kSeg - 1) / kSeg * kSeg; }
constexpr size_t kNoAllocF4 = seg(kNoAllocPaths * sizeof(float4));
constexpr size_t kNoAllocI4 = seg(kNoAllocPaths * sizeof(int32_t));
constexpr size_t kNoAllocCounts = seg((kNoAllocDepth + 2) * kCountStride * sizeof(int32_t));
constexpr size_t kNoAllocTally = seg(16 * sizeof(unsigned long long));
// beta, radiance, q_o[2], q_d[2], hits, s_o, s_d, s_pb: 10 float4 arrays;
// misc, q_slot[2], s_target: 4 int arrays.
constexpr size_t kNoAllocBytes = 10 * kNoAllocF4 + 4 * kNoAllocI4 + kNoAllocCounts + kNoAllocTally;
static_assert(kNoAllocBytes == XYZGPU_NOALLOC_SCRATCH_BYTES,
              "XYZGPU_NOALLOC_SCRATCH_BYTES must match the scratch layout");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mu;

// Per device: the array's device address and the launch grids of the five
// kernels (occupancy x SM count of that device).  An entry is published, under
// g_noalloc_mu, only once all of its fields are set.
struct NoAllocDevice {
  unsigned char *base;
  int raygen, trace_e, trace_s, shade, film;
};
NoAllocDevice g_noalloc_dev[64] = {};

// Set-up of `device` (which must be current): the first call on a device looks
// the symbol up and sizes the grids; later calls reuse them.
int noalloc_device(int device, NoAllocDevice *out) {
  if (device < 0 || device >= 64)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: device ordinal %d is beyond 63", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_dev[device].base) {
    void *p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return set_error(XYZGPU_E_CUDA, "render_noalloc: cudaGetSymbolAddress failed: %s",
                       cudaGetErrorString(e));
    NoAllocDevice d;
    d.raygen = occupancy_grid(k_raygen<false>, device);
    d.trace_e = occupancy_grid(k_trace_queue<false, false>, device);
    d.trace_s = occupancy_grid(k_trace_queue<true, false>, device);
    d.shade = occupancy_grid(k_shade<kModePlain>, device);
    d.film = occupancy_grid(k_film, device);
    d.base = static_cast<unsigned char *>(p);
    g_noalloc_dev[device] = d;
  }
  *out = g_noalloc_dev[device];
  return XYZGPU_OK;
}

}  // namespace

int render_noalloc_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp,
                          float *film, cudaStream_t st) {
  if (rp.film_location != XYZGPU_FILM_DEVICE)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: the film must be device memory");
  if (rp.profile != XYZGPU_PROFILE_OFF)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: profiling is not available");
  if (rp.spectral != XYZGPU_SPECTRAL_OFF)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: only the XYZ film mode is available");
  if (s.dev.has_metal)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: scenes with metal materials are not available");
  if (rp.wave_paths > kNoAllocPaths)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: wave_paths %d exceeds the maximum of %lld",
                     rp.wave_paths, static_cast<long long>(kNoAllocPaths));
  if (rp.max_depth > kNoAllocDepth)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: max_depth %d exceeds the maximum of %d",
                     rp.max_depth, kNoAllocDepth);
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  NoAllocDevice dev;
  int rc = noalloc_device(s.device, &dev);
  if (rc) return rc;
  unsigned char *const base = dev.base;

  WaveArgs A;
  std::memset(&A, 0, sizeof(A));
  unsigned char *p = base;
  auto take = [&p](size_t bytes) {
    unsigned char *q = p;
    p += bytes;
    return q;
  };
  A.beta = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.radiance = reinterpret_cast<float4 *>(take(kNoAllocF4));
  for (int q = 0; q < 2; ++q) {
    A.q_o[q] = reinterpret_cast<float4 *>(take(kNoAllocF4));
    A.q_d[q] = reinterpret_cast<float4 *>(take(kNoAllocF4));
  }
  A.hits = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_o = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_d = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_pb = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.misc = reinterpret_cast<uint32_t *>(take(kNoAllocI4));
  for (int q = 0; q < 2; ++q) A.q_slot[q] = reinterpret_cast<int32_t *>(take(kNoAllocI4));
  A.s_target = reinterpret_cast<int32_t *>(take(kNoAllocI4));
  A.counts = reinterpret_cast<int32_t *>(take(kNoAllocCounts));
  unsigned long long *tally = reinterpret_cast<unsigned long long *>(take(kNoAllocTally));

  A.S = s.dev;
  A.cam = camera_setup(cam, rp.width, rp.height);
  A.W = rp.width;
  A.H = rp.height;
  A.kmax = rp.max_depth + 1;
  A.rr_start = rp.rr_start_depth;
  A.rr_threshold = rp.rr_threshold;
  A.seed = rp.seed;

  int64_t const npix_total = static_cast<int64_t>(rp.width) * rp.height;
  int64_t const cap = rp.wave_paths > 0 ? rp.wave_paths : kNoAllocPaths;
  int const iters = rp.max_depth;
  if (!rp.accumulate) XYZ_CUDA_TRY(cudaMemsetAsync(film, 0, 3 * npix_total * sizeof(float), st));
  XYZ_CUDA_TRY(cudaMemsetAsync(tally, 0, kNoAllocTally, st));
  int64_t const spp_per_wave =
      std::max<int64_t>(1, std::min<int64_t>(rp.spp, cap / std::max<int64_t>(1, npix_total)));
  int64_t const pix_per_wave = std::min<int64_t>(npix_total, cap);
  for (int64_t s0 = 0; s0 < rp.spp; s0 += spp_per_wave) {
    int const ns = static_cast<int>(std::min<int64_t>(spp_per_wave, rp.spp - s0));
    for (int64_t p0 = 0; p0 < npix_total; p0 += pix_per_wave) {
      A.p0 = p0;
      A.npix = std::min<int64_t>(pix_per_wave, npix_total - p0);
      A.s0 = static_cast<uint32_t>(rp.spp_offset + s0);
      A.nsamp = ns;
      A.npaths = A.npix * ns;
      // queue lengths and work counters from the previous wave or call
      XYZ_CUDA_TRY(cudaMemsetAsync(A.counts, 0, kNoAllocCounts, st));
      int const gr = static_cast<int>(std::min<int64_t>(dev.raygen, (A.npaths + kThreads - 1) / kThreads));
      k_raygen<false><<<gr, kThreads, 0, st>>>(A);
      for (int b = 0; b < iters; ++b) {
        k_trace_queue<false, false><<<dev.trace_e, kThreads, 0, st>>>(A, b, tally + 8);
        k_shade<kModePlain><<<dev.shade, kThreads, 0, st>>>(A, b);
        k_trace_queue<true, false><<<dev.trace_s, kThreads, 0, st>>>(A, b, tally + 8);
      }
      int const gf = static_cast<int>(std::min<int64_t>(dev.film, (A.npix + kThreads - 1) / kThreads));
      k_film<<<gf, kThreads, 0, st>>>(A, film);
      XYZ_CUDA_TRY(cudaGetLastError());
    }
  }
  return XYZGPU_OK;
}

}  // namespace xyzgpu
