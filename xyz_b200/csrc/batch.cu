// Batched rendering: xyzgpu_batch_* and xyzgpu_render_batch.
//
// Many scenes share every kernel launch.  The paths of all jobs are laid out as
// blocks (a run of consecutive samples of one job over all of its pixels) that
// are packed greedily into waves of at most `wave_paths` paths; a job's blocks
// appear in sample order, so each film receives its samples in the order of a
// single-scene render and the films are identical to xyzgpu_render's.  The
// kernels are the single-scene wavefront kernels instantiated with kBatch:
// each queue record carries its path's block, from which a kernel reads the
// scene (kd-tree, triangles, materials, lights), the camera and the estimator
// parameters in the device job table.  The traversal kernels are persistent
// (grid = CTAs per SM x SMs, lanes refilled from a work counter); the others
// stride over their queues.
//
// A launch is one CUDA graph whose control flow runs on the device: a start
// kernel (film clears, tally, cursor), then a conditional WHILE node over the
// waves whose body is: wave start (the cursor takes the wave's entry from the
// device wave table, counters cleared), ray generation, a nested WHILE node over
// the bounces (closest hit, shading, shadow rays, bounce end), film and tallies,
// wave end.  The bounce loop ends when the wave's bounces are done or its
// extension queue is empty, the wave loop after the last wave.  The batched
// kernels read the wave and bounce from the device cursor, so the graph has the
// same dozen nodes however many waves the batch has, and the host issues one
// cudaGraphLaunch per batch.  The same kernels issued one by one from the host
// (use_graph = 0, and the autotuner's probes) render the same films.  Sample
// offsets live in the job table and can change between launches without
// re-capture.  The batch owns its path buffers (the graph holds their
// addresses).
//
// Autotuner: coordinate descent over the pixel tile of the slot order (tiles
// make camera rays of neighbouring lanes coherent), the wave size (2^22 to
// 2^27 paths: occupancy of late bounces vs. memory) and the trace grid (CTAs per SM); each candidate is
// timed with CUDA events on this batch (optionally with capped samples) into
// scratch films.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "wavefront.cuh"

namespace xyzgpu {

void free_wave_buffers(RenderWorkspace &w);

namespace {

constexpr int64_t kDefaultBatchWave = int64_t{1} << 24;

using WavePlan = BatchWave;

// Tally words the control kernels count in: waves and bounces run by the launch.
constexpr int kTallyWaves = 3, kTallyBounces = 4;
static_assert(kTallyBounces < kTallyIterBase, "batch tally words");

struct Batch {
  int device = 0;
  std::vector<xyzgpu_batch_job> jobs;
  std::vector<BatchJob> table;
  xyzgpu_batch_config cfg{};
  std::vector<WaveBlock> blocks;
  std::vector<WavePlan> waves;
  BatchJob *d_jobs = nullptr;
  WaveBlock *d_blocks = nullptr;
  size_t d_blocks_cap = 0;
  BatchWave *d_waves = nullptr;
  size_t d_waves_cap = 0;
  BatchCursor *d_cursor = nullptr;
  RenderWorkspace ws;
  unsigned long long *d_tally = nullptr;
  cudaStream_t cap_stream = nullptr;
  cudaStream_t last_stream = nullptr;
  bool launched = false;
  cudaGraphExec_t exec = nullptr;
  int graph_nodes = 0, graph_top_nodes = 0;
  uint64_t paths = 0, launches_per_launch = 0;
  int max_iters = 0;
  int grid_raygen = 0, grid_trace_e = 0, grid_trace_s = 0, grid_shade = 0, grid_film = 0;
};

int job_tile(const Batch &b, size_t j) {
  int const t = b.cfg.tile;
  xyzgpu_render_params const &p = b.jobs[j].params;
  if (t <= 1 || p.width % t != 0 || p.height % t != 0) return 1;
  return t;
}

// Blocks and waves for wave capacity `cap`; spp_cap > 0 limits every job's
// samples (autotuner probes).
int plan_waves(Batch &b, int64_t cap, int spp_cap) {
  b.blocks.clear();
  b.waves.clear();
  b.paths = 0;
  WavePlan cur{};
  int64_t used = 0;
  auto close = [&]() {
    if (cur.n_blocks > 0) b.waves.push_back(cur);
    cur = WavePlan{};
    cur.first_block = static_cast<int>(b.blocks.size());
    used = 0;
  };
  for (size_t j = 0; j < b.jobs.size(); ++j) {
    xyzgpu_render_params const &p = b.jobs[j].params;
    int64_t const npix = static_cast<int64_t>(p.width) * p.height;
    if (npix > cap)
      return set_error(XYZGPU_E_LIMIT, "batch: job %zu has %lld pixels, more than the wave of %lld paths", j,
                       static_cast<long long>(npix), static_cast<long long>(cap));
    int const spp = spp_cap > 0 ? std::min(p.spp, spp_cap) : p.spp;
    int done = 0;
    while (done < spp) {
      int64_t const room = (cap - used) / npix;
      if (room <= 0) {
        close();
        continue;
      }
      int const ns = static_cast<int>(std::min<int64_t>(room, spp - done));
      WaveBlock wb;
      wb.job = static_cast<int>(j);
      wb.ns = ns;
      wb.s0 = static_cast<uint32_t>(done);
      wb.npix = npix;
      wb.slot_off = used;
      wb.pix_off = cur.film_threads;
      b.blocks.push_back(wb);
      cur.n_blocks += 1;
      cur.npaths += npix * ns;
      cur.film_threads += npix;
      cur.iters = std::max(cur.iters, p.max_depth);
      used += npix * ns;
      done += ns;
      b.paths += static_cast<uint64_t>(npix * ns);
    }
  }
  close();
  return XYZGPU_OK;
}

int upload_tables(Batch &b, const std::vector<float *> *films, cudaStream_t st) {
  std::vector<BatchJob> t = b.table;
  for (size_t j = 0; j < t.size(); ++j) {
    t[j].tile = job_tile(b, j);
    t[j].clear = b.jobs[j].params.accumulate ? 0 : 1;
    if (films) t[j].film = (*films)[j];
  }
  XYZ_CUDA_TRY(cudaMemcpyAsync(b.d_jobs, t.data(), t.size() * sizeof(BatchJob), cudaMemcpyHostToDevice, st));
  if (b.waves.size() > b.d_waves_cap) {
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(b.d_waves);
    b.d_waves = nullptr;
    b.d_waves_cap = 0;
    XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&b.d_waves), b.waves.size() * sizeof(BatchWave)));
    b.d_waves_cap = b.waves.size();
  }
  if (!b.waves.empty())
    XYZ_CUDA_TRY(cudaMemcpyAsync(b.d_waves, b.waves.data(), b.waves.size() * sizeof(BatchWave),
                                 cudaMemcpyHostToDevice, st));
  if (b.blocks.size() > b.d_blocks_cap) {
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(b.d_blocks);
    b.d_blocks = nullptr;
    b.d_blocks_cap = 0;
    XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&b.d_blocks), b.blocks.size() * sizeof(WaveBlock)));
    b.d_blocks_cap = b.blocks.size();
  }
  if (!b.blocks.empty())
    XYZ_CUDA_TRY(cudaMemcpyAsync(b.d_blocks, b.blocks.data(), b.blocks.size() * sizeof(WaveBlock),
                                 cudaMemcpyHostToDevice, st));
  // the host vectors are pageable: the copies have completed on return
  return XYZGPU_OK;
}

void set_grids(Batch &b) {
  int const sms = sm_count(b.device);
  b.grid_raygen = occupancy_grid(k_raygen<true>, b.device);
  b.grid_shade = occupancy_grid(k_shade<kModeBatch>, b.device);
  b.grid_film = occupancy_grid(k_film_batch, b.device);
  int const occ_e = occupancy_grid(k_trace_queue<false, false, kModeBatch>, b.device) / sms;
  int const occ_s = occupancy_grid(k_trace_queue<true, false, kModeBatch>, b.device) / sms;
  int const want = b.cfg.trace_ctas_per_sm;
  b.grid_trace_e = (want > 0 ? std::min(want, occ_e) : occ_e) * sms;
  b.grid_trace_s = (want > 0 ? std::min(want, occ_s) : occ_s) * sms;
}

// ------------------------------------------------------- control kernels
// Launch start: the tally is cleared, the films of jobs that do not accumulate
// are zeroed (grid y strides over the jobs) and the cursor goes to wave 0.
__global__ void __launch_bounds__(kThreads) k_batch_begin(const BatchJob *jobs, int n_jobs,
                                                          unsigned long long *tally, BatchCursor *cur) {
  if (blockIdx.x == 0 && blockIdx.y == 0) {
    for (int i = threadIdx.x; i < kTallyWords; i += blockDim.x) tally[i] = 0;
    if (threadIdx.x == 0) {
      cur->wave = 0;
      cur->bounce = 0;
    }
  }
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int j = blockIdx.y; j < n_jobs; j += gridDim.y) {
    BatchJob const &J = jobs[j];
    if (!J.clear) continue;
    int64_t const n = 3 * static_cast<int64_t>(J.W) * J.H;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
      J.film[i] = 0.0f;
  }
}

// Wave start: the cursor takes the entry of its wave and bounce 0; the wave's
// queue counters are cleared.  In a graph it also opens the bounce loop.
template <bool kGraph>
__global__ void k_batch_wave_begin(const BatchWave *waves, BatchCursor *cur, int32_t *counts,
                                   cudaGraphConditionalHandle bounce_loop) {
  BatchWave const w = waves[cur->wave];
  int const nc = (w.iters + 2) * kCountStride;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) counts[i] = 0;
  if (threadIdx.x == 0) {
    cur->w = w;
    cur->bounce = 0;
    if constexpr (kGraph) cudaGraphSetConditional(bounce_loop, w.iters > 0 ? 1u : 0u);
  }
}

// Bounce end: the cursor moves to the next bounce, which runs (in a graph)
// while the wave has bounces left and rays in its extension queue.
template <bool kGraph>
__global__ void k_batch_bounce_end(BatchCursor *cur, const int32_t *counts, unsigned long long *tally,
                                   cudaGraphConditionalHandle bounce_loop) {
  int const b = cur->bounce + 1;
  cur->bounce = b;
  tally[kTallyBounces] += 1;
  if constexpr (kGraph) {
    bool const more = b < cur->w.iters && counts[b * kCountStride + kCExt] > 0;
    cudaGraphSetConditional(bounce_loop, more ? 1u : 0u);
  }
}

// Wave end: the cursor moves to the next wave; the wave loop (in a graph)
// ends after the last one.
template <bool kGraph>
__global__ void k_batch_wave_end(BatchCursor *cur, int n_waves, unsigned long long *tally,
                                 cudaGraphConditionalHandle wave_loop) {
  int const w = cur->wave + 1;
  cur->wave = w;
  tally[kTallyWaves] += 1;
  if constexpr (kGraph) cudaGraphSetConditional(wave_loop, w < n_waves ? 1u : 0u);
}

WaveArgs wave_args(const Batch &b) {
  WaveArgs A;
  std::memset(&A, 0, sizeof(A));
  RenderWorkspace const &wv = b.ws;
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
  A.fsn = wv.fsn;
  A.s_slot = wv.s_slot;
  A.hero = 1;
  A.jobs = b.d_jobs;
  A.blocks = b.d_blocks;
  A.cursor = b.d_cursor;
  return A;
}

dim3 begin_grid(const Batch &b) {
  return dim3(static_cast<unsigned>(std::max(1, sm_count(b.device))),
              static_cast<unsigned>(std::min<size_t>(b.jobs.size(), 65535)));
}

// Issues the launch from the host, kernel by kernel, on `st`: the start
// kernel, then every wave of the plan with all of its bounces.  The films are
// the job table's (the autotuner points them at scratch films).
int issue(Batch &b, cudaStream_t st) {
  WaveArgs const A = wave_args(b);
  int const n_waves = static_cast<int>(b.waves.size());
  k_batch_begin<<<begin_grid(b), kThreads, 0, st>>>(b.d_jobs, static_cast<int>(b.jobs.size()), b.d_tally,
                                                     b.d_cursor);
  uint64_t launches = 1;
  for (WavePlan const &w : b.waves) {
    k_batch_wave_begin<false><<<1, kThreads, 0, st>>>(b.d_waves, b.d_cursor, b.ws.counts, 0);
    k_raygen<true><<<b.grid_raygen, kThreads, 0, st>>>(A);
    for (int it = 0; it < w.iters; ++it) {
      k_trace_queue<false, false, kModeBatch><<<b.grid_trace_e, kThreads, 0, st>>>(A, it, nullptr);
      k_shade<kModeBatch><<<b.grid_shade, kThreads, 0, st>>>(A, it);
      k_trace_queue<true, false, kModeBatch><<<b.grid_trace_s, kThreads, 0, st>>>(A, it, nullptr);
      k_batch_bounce_end<false><<<1, 1, 0, st>>>(b.d_cursor, b.ws.counts, b.d_tally, 0);
    }
    k_film_batch<<<b.grid_film, kThreads, 0, st>>>(A);
    k_tally<<<1, 32, 0, st>>>(A, 0, b.d_tally);
    k_batch_wave_end<false><<<1, 1, 0, st>>>(b.d_cursor, n_waves, b.d_tally, 0);
    launches += 5 + 4 * static_cast<uint64_t>(w.iters);
    XYZ_CUDA_TRY(cudaGetLastError());
  }
  b.launches_per_launch = launches;
  return XYZGPU_OK;
}

void drop_graph(Batch &b) {
  if (b.exec) cudaGraphExecDestroy(b.exec);
  b.exec = nullptr;
  b.graph_nodes = b.graph_top_nodes = 0;
}

size_t node_count(cudaGraph_t g) {
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  return n;
}

// Captures `emit`'s launches on the capture stream into `g` after `deps`
// (ndeps of them) and returns the last node captured in *last.
template <class F>
cudaError_t capture_into(cudaStream_t cs, cudaGraph_t g, const cudaGraphNode_t *deps, size_t ndeps, F &&emit,
                         cudaGraphNode_t *last) {
  cudaError_t e = cudaStreamBeginCaptureToGraph(cs, g, deps, nullptr, ndeps, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  emit();
  cudaError_t const le = cudaGetLastError();
  cudaStreamCaptureStatus status;
  const cudaGraphNode_t *tail = nullptr;
  size_t ntail = 0;
  e = cudaStreamGetCaptureInfo(cs, &status, nullptr, nullptr, &tail, &ntail);
  cudaGraphNode_t const t = (e == cudaSuccess && ntail == 1) ? tail[0] : nullptr;
  cudaGraph_t out = nullptr;
  cudaError_t const ee = cudaStreamEndCapture(cs, &out);
  if (le != cudaSuccess) return le;
  if (e != cudaSuccess) return e;
  if (ee != cudaSuccess) return ee;
  if (!t) return cudaErrorStreamCaptureUnjoined;
  *last = t;
  return cudaSuccess;
}

// Adds a WHILE node after `dep` to `g` and returns its body graph.
cudaError_t add_while(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h, cudaGraphNode_t *node,
                      cudaGraph_t *body) {
  cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaError_t const e = cudaGraphAddNode(node, g, &dep, 1, &p);
  if (e != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  return cudaSuccess;
}

// Builds the launch graph: start kernel -> WHILE(waves) { wave start, ray
// generation -> WHILE(bounces) { closest hit, shading, shadow rays, bounce
// end } -> film, tally, wave end }.
int capture(Batch &b) {
  drop_graph(b);
  if (!b.cfg.use_graph) return XYZGPU_OK;
  if (!b.cap_stream) XYZ_CUDA_TRY(cudaStreamCreateWithFlags(&b.cap_stream, cudaStreamNonBlocking));
  cudaStream_t const cs = b.cap_stream;
  WaveArgs const A = wave_args(b);
  int const n_waves = static_cast<int>(b.waves.size());
  int const n_jobs = static_cast<int>(b.jobs.size());
  cudaGraph_t g = nullptr;
  XYZ_CUDA_TRY(cudaGraphCreate(&g, 0));
  cudaError_t e = cudaSuccess;
  cudaGraphConditionalHandle wave_loop = 0, bounce_loop = 0;
  cudaGraphNode_t n_begin = nullptr, n_waves_node = nullptr, n_raygen = nullptr, n_bounces = nullptr,
                  n_tail = nullptr;
  cudaGraph_t wave_body = nullptr, bounce_body = nullptr;
  do {
    e = cudaGraphConditionalHandleCreate(&wave_loop, g, n_waves > 0 ? 1u : 0u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) break;
    e = capture_into(cs, g, nullptr, 0, [&] {
      k_batch_begin<<<begin_grid(b), kThreads, 0, cs>>>(b.d_jobs, n_jobs, b.d_tally, b.d_cursor);
    }, &n_begin);
    if (e != cudaSuccess) break;
    e = add_while(g, n_begin, wave_loop, &n_waves_node, &wave_body);
    if (e != cudaSuccess) break;
    e = cudaGraphConditionalHandleCreate(&bounce_loop, wave_body, 0u, 0u);
    if (e != cudaSuccess) break;
    e = capture_into(cs, wave_body, nullptr, 0, [&] {
      k_batch_wave_begin<true><<<1, kThreads, 0, cs>>>(b.d_waves, b.d_cursor, b.ws.counts, bounce_loop);
      k_raygen<true><<<b.grid_raygen, kThreads, 0, cs>>>(A);
    }, &n_raygen);
    if (e != cudaSuccess) break;
    e = add_while(wave_body, n_raygen, bounce_loop, &n_bounces, &bounce_body);
    if (e != cudaSuccess) break;
    e = capture_into(cs, bounce_body, nullptr, 0, [&] {
      k_trace_queue<false, false, kModeBatch><<<b.grid_trace_e, kThreads, 0, cs>>>(A, 0, nullptr);
      k_shade<kModeBatch><<<b.grid_shade, kThreads, 0, cs>>>(A, 0);
      k_trace_queue<true, false, kModeBatch><<<b.grid_trace_s, kThreads, 0, cs>>>(A, 0, nullptr);
      k_batch_bounce_end<true><<<1, 1, 0, cs>>>(b.d_cursor, b.ws.counts, b.d_tally, bounce_loop);
    }, &n_tail);
    if (e != cudaSuccess) break;
    e = capture_into(cs, wave_body, &n_bounces, 1, [&] {
      k_film_batch<<<b.grid_film, kThreads, 0, cs>>>(A);
      k_tally<<<1, 32, 0, cs>>>(A, 0, b.d_tally);
      k_batch_wave_end<true><<<1, 1, 0, cs>>>(b.d_cursor, n_waves, b.d_tally, wave_loop);
    }, &n_tail);
  } while (false);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_error(XYZGPU_E_CUDA, "batch: building the launch graph failed: %s", cudaGetErrorString(e));
  }
  size_t const top = node_count(g);
  size_t const nodes = top + node_count(wave_body) + node_count(bounce_body);
  cudaError_t const e2 = cudaGraphInstantiate(&b.exec, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) {
    b.exec = nullptr;
    return set_error(XYZGPU_E_CUDA, "batch: graph instantiation failed: %s", cudaGetErrorString(e2));
  }
  b.graph_nodes = static_cast<int>(nodes);
  b.graph_top_nodes = static_cast<int>(top);
  return XYZGPU_OK;
}

// Plans waves, sizes the path buffers and uploads the tables for b.cfg.
int prepare(Batch &b, int spp_cap, const std::vector<float *> *films, cudaStream_t st) {
  int64_t total = 0, max_pix = 1;
  for (auto const &j : b.jobs) {
    int64_t const npix = static_cast<int64_t>(j.params.width) * j.params.height;
    int const spp = spp_cap > 0 ? std::min(j.params.spp, spp_cap) : j.params.spp;
    total += npix * spp;
    max_pix = std::max(max_pix, npix);
  }
  if (b.cfg.wave_paths > 0 && b.cfg.wave_paths < max_pix)
    return set_error(XYZGPU_E_LIMIT, "batch: wave of %d paths is smaller than the largest image (%lld pixels)",
                     b.cfg.wave_paths, static_cast<long long>(max_pix));
  int64_t cap = b.cfg.wave_paths > 0 ? b.cfg.wave_paths : std::min(total, kDefaultBatchWave);
  cap = std::max(cap, max_pix);
  b.cfg.wave_paths = static_cast<int>(std::min<int64_t>(cap, INT32_MAX));
  int rc = plan_waves(b, cap, spp_cap);
  if (rc) return rc;
  rc = ensure_wave_buffers(b.ws, cap, b.max_iters);
  if (rc) return rc;
  set_grids(b);
  return upload_tables(b, films, st);
}

}  // namespace
}  // namespace xyzgpu

using namespace xyzgpu;

struct xyzgpu_batch_s {
  Batch b;
};

extern "C" {

void xyzgpu_batch_config_default(xyzgpu_batch_config *cfg) {
  if (!cfg) return;
  cfg->wave_paths = 0;
  cfg->tile = 1;
  cfg->trace_ctas_per_sm = 0;
  cfg->use_graph = 1;
}

void xyzgpu_batch_destroy(xyzgpu_batch h) {
  if (!h) return;
  Batch &b = h->b;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b.device);
  cudaDeviceSynchronize();
  drop_graph(b);
  if (b.cap_stream) cudaStreamDestroy(b.cap_stream);
  cudaFree(b.d_jobs);
  cudaFree(b.d_blocks);
  cudaFree(b.d_waves);
  cudaFree(b.d_cursor);
  cudaFree(b.d_tally);
  free_wave_buffers(b.ws);
  cudaSetDevice(prev);
  delete h;
}

int xyzgpu_batch_create(const xyzgpu_batch_job *jobs, int n_jobs, const xyzgpu_batch_config *cfg,
                        xyzgpu_batch *out) {
  clear_error();
  if (!jobs || !out || n_jobs <= 0) return set_error(XYZGPU_E_INVALID, "batch_create: no jobs");
  *out = nullptr;
  xyzgpu_batch_config c;
  if (cfg)
    c = *cfg;
  else
    xyzgpu_batch_config_default(&c);
  if (c.wave_paths < 0 || c.tile < 0 || c.tile > 64 || c.trace_ctas_per_sm < 0)
    return set_error(XYZGPU_E_INVALID, "batch_create: configuration out of range");
  if (c.tile == 0) c.tile = 1;
  auto *scene0 = reinterpret_cast<SceneImpl *>(jobs[0].scene);
  for (int j = 0; j < n_jobs; ++j) {
    xyzgpu_batch_job const &J = jobs[j];
    xyzgpu_render_params const &p = J.params;
    if (!J.scene || !J.film) return set_error(XYZGPU_E_INVALID, "batch_create: job %d: null scene or film", j);
    if (reinterpret_cast<uintptr_t>(J.film) & 3u)
      return set_error(XYZGPU_E_INVALID, "batch_create: job %d: film must be 4-byte aligned", j);
    if (reinterpret_cast<SceneImpl *>(J.scene)->device != scene0->device)
      return set_error(XYZGPU_E_INVALID, "batch_create: job %d: scenes must be on one device", j);
    if (p.width <= 0 || p.height <= 0 || p.spp < 0 || p.spp_offset < 0 || p.max_depth < 1 ||
        p.max_depth > 1000 || p.rr_start_depth < 1 || !(p.rr_threshold >= 0.0f))
      return set_error(XYZGPU_E_INVALID, "batch_create: job %d: parameters out of range", j);
    if (p.spectral != XYZGPU_SPECTRAL_OFF || p.profile != XYZGPU_PROFILE_OFF || p.row_begin != 0 || p.row_end != 0)
      return set_error(XYZGPU_E_INVALID, "batch_create: job %d: XYZ film mode, whole images, no profiling", j);
    if (static_cast<int64_t>(p.width) * p.height >= (1ll << 31))
      return set_error(XYZGPU_E_LIMIT, "batch_create: job %d: image exceeds 2^31 pixels", j);
    if (static_cast<int64_t>(p.spp_offset) + p.spp >= (1ll << 32))
      return set_error(XYZGPU_E_LIMIT, "batch_create: job %d: sample index exceeds 2^32", j);
    xyzgpu_camera const &cam = J.camera;
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(cam.eye[k]) || !std::isfinite(cam.at[k]))
        return set_error(XYZGPU_E_INVALID, "batch_create: job %d: camera position is not finite", j);
    if (!(cam.film_size > 0) || !(cam.focal_length > 0) || !(cam.f_number > 0))
      return set_error(XYZGPU_E_INVALID, "batch_create: job %d: camera film size, focal length and F-number must be > 0", j);
  }
  auto *h = new (std::nothrow) xyzgpu_batch_s();
  if (!h) return set_error(XYZGPU_E_NOMEM, "batch_create: host allocation failed");
  Batch &b = h->b;
  b.device = scene0->device;
  b.cfg = c;
  b.jobs.assign(jobs, jobs + n_jobs);
  b.table.resize(n_jobs);
  for (int j = 0; j < n_jobs; ++j) {
    xyzgpu_batch_job const &J = jobs[j];
    BatchJob &t = b.table[j];
    std::memset(&t, 0, sizeof(t));
    t.S = reinterpret_cast<SceneImpl *>(J.scene)->dev;
    t.cam = camera_setup(J.camera, J.params.width, J.params.height);
    t.W = J.params.width;
    t.H = J.params.height;
    t.kmax = J.params.max_depth + 1;
    t.rr_start = J.params.rr_start_depth;
    t.rr_threshold = J.params.rr_threshold;
    t.tile = 1;
    t.seed = J.params.seed;
    t.spp_offset = static_cast<uint32_t>(J.params.spp_offset);
    t.film = J.film;
    b.max_iters = std::max(b.max_iters, J.params.max_depth);
  }
  auto fail = [&](int rc) {
    xyzgpu_batch_destroy(h);
    return rc;
  };
  if (cudaSetDevice(b.device) != cudaSuccess) return fail(set_error(XYZGPU_E_CUDA, "batch_create: cudaSetDevice failed"));
  if (cudaMalloc(reinterpret_cast<void **>(&b.d_jobs), n_jobs * sizeof(BatchJob)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&b.d_tally), kTallyWords * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&b.d_cursor), sizeof(BatchCursor)) != cudaSuccess)
    return fail(set_error(XYZGPU_E_NOMEM, "batch_create: allocating the job table failed"));
  int rc = prepare(b, 0, nullptr, nullptr);
  if (rc) return fail(rc);
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) return fail(set_error(XYZGPU_E_CUDA, "batch_create: upload failed"));
  rc = capture(b);
  if (rc) return fail(rc);
  *out = h;
  return XYZGPU_OK;
}

int xyzgpu_batch_launch(xyzgpu_batch h, void *stream) {
  clear_error();
  if (!h) return set_error(XYZGPU_E_INVALID, "batch_launch: null batch");
  Batch &b = h->b;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(b.device));
  if (b.exec) {
    XYZ_CUDA_TRY(cudaGraphLaunch(b.exec, st));
  } else {
    int const rc = issue(b, st);
    if (rc) return rc;
  }
  b.last_stream = st;
  b.launched = true;
  return XYZGPU_OK;
}

int xyzgpu_batch_set_sample_offsets(xyzgpu_batch h, const uint32_t *offsets) {
  clear_error();
  if (!h || !offsets) return set_error(XYZGPU_E_INVALID, "batch_set_sample_offsets: null argument");
  Batch &b = h->b;
  for (size_t j = 0; j < b.jobs.size(); ++j)
    if (static_cast<uint64_t>(offsets[j]) + b.jobs[j].params.spp >= (1ull << 32))
      return set_error(XYZGPU_E_LIMIT, "batch_set_sample_offsets: job %zu: sample index exceeds 2^32", j);
  XYZ_CUDA_TRY(cudaSetDevice(b.device));
  // the next launch reads the table; launches in flight must not see it change
  if (b.launched) XYZ_CUDA_TRY(cudaStreamSynchronize(b.last_stream));
  for (size_t j = 0; j < b.jobs.size(); ++j) {
    b.jobs[j].params.spp_offset = static_cast<int>(offsets[j]);
    b.table[j].spp_offset = offsets[j];
  }
  int const rc = upload_tables(b, nullptr, nullptr);
  if (rc) return rc;
  XYZ_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return XYZGPU_OK;
}

int xyzgpu_batch_autotune(xyzgpu_batch h, int trials, int probe_spp, void *stream,
                          xyzgpu_batch_config *chosen) {
  clear_error();
  if (!h || trials < 1 || probe_spp < 0) return set_error(XYZGPU_E_INVALID, "batch_autotune: bad argument");
  Batch &b = h->b;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(b.device));
  if (b.launched) XYZ_CUDA_TRY(cudaStreamSynchronize(b.last_stream));
  drop_graph(b);
  // scratch films so the callers' films are untouched
  size_t total_film = 0;
  for (auto const &j : b.jobs) total_film += 3 * static_cast<size_t>(j.params.width) * j.params.height;
  float *scratch = nullptr;
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&scratch), total_film * sizeof(float)));
  std::vector<float *> films(b.jobs.size());
  {
    size_t off = 0;
    for (size_t j = 0; j < b.jobs.size(); ++j) {
      films[j] = scratch + off;
      off += 3 * static_cast<size_t>(b.jobs[j].params.width) * b.jobs[j].params.height;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = XYZGPU_OK;
  auto time_cfg = [&](const xyzgpu_batch_config &c, float *ms) -> int {
    b.cfg = c;
    int r = prepare(b, probe_spp, &films, st);
    if (r) return r;
    float best = INFINITY;
    for (int t = 0; t < trials + 1; ++t) {  // the first run warms up
      XYZ_CUDA_TRY(cudaEventRecord(e0, st));
      r = issue(b, st);
      if (r) return r;
      XYZ_CUDA_TRY(cudaEventRecord(e1, st));
      XYZ_CUDA_TRY(cudaEventSynchronize(e1));
      float m = 0.0f;
      XYZ_CUDA_TRY(cudaEventElapsedTime(&m, e0, e1));
      if (t > 0) best = std::min(best, m);
    }
    *ms = best;
    return XYZGPU_OK;
  };
  do {
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      rc = set_error(XYZGPU_E_CUDA, "batch_autotune: event creation failed");
      break;
    }
    int64_t total = 0, max_pix = 1;
    for (auto const &j : b.jobs) {
      int64_t const npix = static_cast<int64_t>(j.params.width) * j.params.height;
      total += npix * (probe_spp > 0 ? std::min(j.params.spp, probe_spp) : j.params.spp);
      max_pix = std::max(max_pix, npix);
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    int64_t const afford = static_cast<int64_t>(free_b / 2) / kBytesPerPath + b.ws.capacity;
    xyzgpu_batch_config best = b.cfg;
    if (best.wave_paths <= 0) best.wave_paths = static_cast<int>(std::max(max_pix, std::min(total, kDefaultBatchWave)));
    float best_ms = 0.0f;
    rc = time_cfg(best, &best_ms);
    if (rc) break;
    int const occ = occupancy_grid(k_trace_queue<false, false, kModeBatch>, b.device) / sm_count(b.device);
    std::vector<int> tiles = {1, 4, 8, 16};
    std::vector<int> waves;
    for (int64_t w = int64_t{1} << 22; w <= (int64_t{1} << 27); w <<= 1)
      if (w >= max_pix && w <= afford && w / 2 < total) waves.push_back(static_cast<int>(w));
    std::vector<int> ctas = {occ, std::max(1, occ * 2 / 3), std::max(1, occ / 2)};
    for (int knob = 0; knob < 3 && rc == XYZGPU_OK; ++knob) {
      std::vector<int> const &vals = knob == 0 ? tiles : (knob == 1 ? waves : ctas);
      xyzgpu_batch_config base = best;
      for (int v : vals) {
        xyzgpu_batch_config c = base;
        if (knob == 0) c.tile = v;
        if (knob == 1) c.wave_paths = v;
        if (knob == 2) c.trace_ctas_per_sm = v;
        if (std::memcmp(&c, &base, sizeof(c)) == 0) continue;
        float ms = 0.0f;
        rc = time_cfg(c, &ms);
        if (rc) break;
        if (ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
    }
    if (rc) break;
    b.cfg = best;
  } while (false);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaFree(scratch);
  if (rc) {
    prepare(b, 0, nullptr, st);
    cudaStreamSynchronize(st);
    capture(b);
    return rc;
  }
  // keep the chosen wave's buffers only
  free_wave_buffers(b.ws);
  rc = prepare(b, 0, nullptr, st);
  if (rc) return rc;
  XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  rc = capture(b);
  if (rc) return rc;
  if (chosen) *chosen = b.cfg;
  return XYZGPU_OK;
}

int xyzgpu_batch_stats_get(xyzgpu_batch h, xyzgpu_batch_stats *out) {
  clear_error();
  if (!h || !out) return set_error(XYZGPU_E_INVALID, "batch_stats_get: null argument");
  Batch &b = h->b;
  XYZ_CUDA_TRY(cudaSetDevice(b.device));
  if (b.launched) XYZ_CUDA_TRY(cudaStreamSynchronize(b.last_stream));
  unsigned long long t[kTallyWords];
  XYZ_CUDA_TRY(cudaMemcpy(t, b.d_tally, sizeof(t), cudaMemcpyDeviceToHost));
  out->paths = b.paths;
  out->waves = b.waves.size();
  // kernels of the last launch: the start kernel, 5 per wave and 4 per bounce
  // (the bounce loop of a graph launch ends early when a wave runs out of rays)
  out->kernel_launches_per_launch =
      b.launched ? 1 + 5 * t[kTallyWaves] + 4 * t[kTallyBounces] : b.launches_per_launch;
  out->extension_rays = b.launched ? t[0] : 0;
  out->shadow_rays = b.launched ? t[1] : 0;
  out->device_bytes = b.ws.capacity * kBytesPerPath +
                      static_cast<int64_t>(b.jobs.size() * sizeof(BatchJob) + b.d_blocks_cap * sizeof(WaveBlock));
  out->graph_nodes = b.graph_nodes;
  out->graph_top_nodes = b.graph_top_nodes;
  return XYZGPU_OK;
}

int xyzgpu_batch_config_get(xyzgpu_batch h, xyzgpu_batch_config *out) {
  clear_error();
  if (!h || !out) return set_error(XYZGPU_E_INVALID, "batch_config_get: null argument");
  *out = h->b.cfg;
  return XYZGPU_OK;
}

int xyzgpu_render_batch(const xyzgpu_batch_job *jobs, int n_jobs, const xyzgpu_batch_config *cfg,
                        void *stream) {
  xyzgpu_batch h = nullptr;
  xyzgpu_batch_config c;
  if (cfg)
    c = *cfg;
  else
    xyzgpu_batch_config_default(&c);
  c.use_graph = 0;  // one launch: nothing to replay
  int rc = xyzgpu_batch_create(jobs, n_jobs, &c, &h);
  if (rc) return rc;
  rc = xyzgpu_batch_launch(h, stream);
  if (!rc && cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess)
    rc = set_error(XYZGPU_E_CUDA, "render_batch: launch failed");
  xyzgpu_batch_destroy(h);
  return rc;
}

}  // extern "C"
