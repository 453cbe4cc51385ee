// Learned path guide: a small MLP that maps a surface point (position,
// normal) to an 8-lobe von Mises-Fisher mixture over directions, trained
// online on the tracer's own radiance samples (xyzgpu_guide_*).
//
// Network: one-blob encoding (Mueller et al., "Neural Importance Sampling",
// 2019) of the 6 inputs into 32 Gaussian bins each (192 values), then
// 192 -> 64 -> 64 -> 64 -> 64 -> 64 with ReLU after the four hidden layers;
// outputs 0..7 are mixture logits, 8..15 log concentrations (clamped to
// [-5, 8]), 16..39 unnormalised lobe means (8 x 3), 40..63 unused.
//
// Arithmetic: bf16 weights and activations, fp32 accumulation, on the 5th
// generation tensor cores: every layer of a tile of 128 rows is a chain of
// tcgen05.mma (M = 128, N = 64, K = 16 each) with both operands in shared
// memory and the accumulator in TMEM; the epilogue (bias, ReLU, bf16 pack)
// reads the accumulator back with tcgen05.ld, one TMEM lane per thread = one
// row.  Training runs the forward pass, the loss gradient at the output, and
// the backward pass on the same tensor cores: the input deltas of a layer
// (delta * W, M = 128) and the weight gradients (delta^T * activations,
// M = 64, N = 64 or 192, reduced over the 128 rows) accumulate in TMEM over
// all tiles a CTA processes (persistent CTAs, 512 TMEM columns), so the
// per-tile weight gradient never leaves the SM; one atomic add per weight
// and CTA at the end.  Adam updates fp32 master weights and re-packs the bf16
// copy.  Operand layouts: tc.cuh.
//
// Loss (per record: point, sampled direction w, weight F / q): the
// importance-sampling estimate of the KL divergence between the normalised
// target F and the mixture p, -F/q * log p(w); its gradient with respect to
// the outputs is written in closed form below (log-sum-exp over lobes).
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "scene.h"
#include "tc.cuh"

namespace xyzgpu {
namespace {

constexpr int kBins = 32;
constexpr int kIn = 6 * kBins;  // 192
constexpr int kW = 64;          // hidden and output width
constexpr int kLayers = 5;
constexpr int kRows = 128;
constexpr int kGuideThreads = 128;
constexpr int kParams = XYZGPU_GUIDE_PARAMS;
constexpr uint32_t kWaitLimit = 1u << 22;

__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kW; }
// flat fp32 parameters: W_l as [K_l][64] row-major, then b_l[64]
__host__ __device__ constexpr int param_w(int l) {
  return l == 0 ? 0 : (kIn * kW + kW) + (l - 1) * (kW * kW + kW);
}
__host__ __device__ constexpr int param_b(int l) { return param_w(l) + layer_in(l) * kW; }
static_assert(param_b(4) + kW == kParams, "parameter count");
// blocked bf16 W^T per layer (64 rows x K_l columns)
__host__ __device__ constexpr uint32_t wblk_off(int l) {
  return l == 0 ? 0u : static_cast<uint32_t>(kW * kIn * 2 + (l - 1) * kW * kW * 2);
}
constexpr uint32_t kWBlkBytes = kW * kIn * 2 + 4 * kW * kW * 2;  // 57344

// TMEM columns: [0, 64) the working accumulator; weight gradients (M = 64
// layout: rows 16w..16w+15 in lanes 32w..32w+15) of layer 0 at [64, 256),
// layers 1..4 at 256 + 64 (l - 1).
__device__ __forceinline__ uint32_t dw_col(int l) { return l == 0 ? 64u : 256u + 64u * (l - 1); }

struct __align__(128) GuideSmem {
  uint8_t w[kWBlkBytes];
  float bias[kLayers][kW];
  uint8_t x[kRows * kIn * 2];
  uint8_t h[4][kRows * kW * 2];
  uint8_t d[2][kRows * kW * 2];
  float db[kLayers][kW];
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};

struct GuideDev {
  const uint8_t *wblk;  // blocked bf16 weights
  const float *params;  // fp32 master (biases read from here)
  float lo[3], inv_ext[3];  // position normalisation: s = (p - lo) * inv_ext
  int *err;
};

// ---------------------------------------------------------------- encoding
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 const v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void store_row8(uint8_t *buf, int r, int c, int cols, const float *v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(buf + tc::blocked_offset(r, c, cols)) = q;
}

// One-blob value of bin j for s in [0, 1]: exp(-(s - (j + 1/2) / 32)^2 / (2 sigma^2)), sigma = 1/32.
__device__ __forceinline__ float blob(float s, int j) {
  float const d = s - (static_cast<float>(j) + 0.5f) * (1.0f / kBins);
  return expf(-d * d * (0.5f * kBins * kBins));
}

// Writes row r of the input encoding from a raw point (position, normal).
__device__ void encode_row(GuideSmem &S, const GuideDev &G, int r, const float f[6]) {
#pragma unroll 1
  for (int dim = 0; dim < 6; ++dim) {
    float s = dim < 3 ? (f[dim] - G.lo[dim]) * G.inv_ext[dim] : (f[dim] + 1.0f) * 0.5f;
    s = fminf(fmaxf(s, 0.0f), 1.0f);
#pragma unroll
    for (int j8 = 0; j8 < kBins; j8 += 8) {
      float v[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) v[t] = blob(s, j8 + t);
      store_row8(S.x, r, dim * kBins + j8, kIn, v);
    }
  }
}

// ---------------------------------------------------------------- stages
__device__ __forceinline__ void publish() {
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
}

// Waits for the committed MMAs; false (uniformly) if any thread gave up,
// in which case `phase` still names the pending completion.
__device__ __forceinline__ bool await_mma(GuideSmem &S, uint32_t &phase) {
  bool const ok = tc::mbar_wait(tc::smem_addr(&S.mbar), phase, kWaitLimit);
  tc::fence_after_sync();
  int const bad = __syncthreads_or(ok ? 0 : 1);
  if (bad) return false;
  phase ^= 1u;
  return true;
}

__device__ __forceinline__ void issue_forward(GuideSmem &S, int l, const uint8_t *in) {
  int const K = layer_in(l);
  uint32_t const a0 = tc::smem_addr(in), b0 = tc::smem_addr(S.w) + wblk_off(l);
  uint32_t const id = tc::idesc_bf16(kRows, kW, false, false);
  for (int ks = 0; ks < K / 16; ++ks)
    tc::mma_bf16(S.tmem, tc::desc_kmajor(a0 + ks * 256, K), tc::desc_kmajor(b0 + ks * 256, K), id, ks > 0);
}

// This thread's row of the working accumulator (64 fp32).
__device__ __forceinline__ void read_acc(const GuideSmem &S, float *v) {
  uint32_t const taddr = S.tmem + ((threadIdx.x & ~31u) << 16);
#pragma unroll
  for (int c = 0; c < kW; c += 16) tc::tmem_ld16(taddr + c, v + c);
  tc::tmem_wait_ld();
}

// Forward pass of the tile whose encoding is in S.x; leaves this thread's
// row of raw outputs (with bias) in out[64].  keep: hidden layers go to
// S.h[0..3] (training), else ping-pong in S.h[0], S.h[1].
__device__ bool forward_tile(GuideSmem &S, uint32_t &phase, bool keep, float *out) {
  int const r = threadIdx.x;
  const uint8_t *in = S.x;
  for (int l = 0; l < kLayers; ++l) {
    publish();
    if (threadIdx.x == 0) {
      tc::fence_after_sync();
      issue_forward(S, l, in);
      tc::mma_commit(tc::smem_addr(&S.mbar));
    }
    if (!await_mma(S, phase)) return false;
    float v[kW];
    read_acc(S, v);
    if (l == kLayers - 1) {
#pragma unroll
      for (int j = 0; j < kW; ++j) out[j] = v[j] + S.bias[l][j];
      break;
    }
    uint8_t *dst = keep ? S.h[l] : S.h[l & 1];
#pragma unroll
    for (int j = 0; j < kW; ++j) v[j] = fmaxf(v[j] + S.bias[l][j], 0.0f);
#pragma unroll
    for (int c = 0; c < kW; c += 8) store_row8(dst, r, c, kW, v + c);
    in = dst;
  }
  return true;
}

// ------------------------------------------------------------- loss gradient
// Mixture of the outputs: weights softmax(o[0..7]), kappa = exp(clamp(o[8+i])),
// means normalise(o[16+3i..]).  log vMF(w) = log k - log 2pi - log(1 - e^-2k) + k (mu.w - 1).
struct Lobes {
  float logpi[8], kappa[8], mu[8][3], len[8], dot[8], logv[8];
  bool clamped[8];
};

__device__ void lobes_from_outputs(const float *o, const float w[3], Lobes &L) {
  float mx = o[0];
  for (int i = 1; i < 8; ++i) mx = fmaxf(mx, o[i]);
  float se = 0.0f;
  for (int i = 0; i < 8; ++i) se += expf(o[i] - mx);
  float const lse = mx + logf(se);
  for (int i = 0; i < 8; ++i) {
    L.logpi[i] = o[i] - lse;
    float lk = o[8 + i];
    L.clamped[i] = lk < -5.0f || lk > 8.0f;
    lk = fminf(fmaxf(lk, -5.0f), 8.0f);
    float const k = expf(lk);
    L.kappa[i] = k;
    float const mx3 = o[16 + 3 * i], my = o[17 + 3 * i], mz = o[18 + 3 * i];
    float const len = sqrtf(mx3 * mx3 + my * my + mz * mz + 1e-12f);
    L.len[i] = len;
    L.mu[i][0] = mx3 / len;
    L.mu[i][1] = my / len;
    L.mu[i][2] = mz / len;
    float const d = L.mu[i][0] * w[0] + L.mu[i][1] * w[1] + L.mu[i][2] * w[2];
    L.dot[i] = d;
    L.logv[i] = lk - 1.8378770664093453f - logf(-expm1f(-2.0f * k)) + k * (d - 1.0f);
  }
}

// d(-scale * log p(w)) / d outputs, into g[0..63].
__device__ void loss_grad(const float *o, const float w[3], float scale, float *g) {
  Lobes L;
  lobes_from_outputs(o, w, L);
  float s[8], mx = -INFINITY;
  for (int i = 0; i < 8; ++i) {
    s[i] = L.logpi[i] + L.logv[i];
    mx = fmaxf(mx, s[i]);
  }
  float se = 0.0f;
  for (int i = 0; i < 8; ++i) se += expf(s[i] - mx);
  float const logp = mx + logf(se);
  for (int j = 0; j < kW; ++j) g[j] = 0.0f;
  for (int i = 0; i < 8; ++i) {
    float const r = expf(s[i] - logp);
    float const pi = expf(L.logpi[i]);
    float const k = L.kappa[i];
    g[i] = -scale * (r - pi);
    // d log v / d log k = 1 - 2k / (e^{2k} - 1) + k (mu.w - 1)
    float const dlk = L.clamped[i] ? 0.0f : r * (1.0f - 2.0f * k / expm1f(2.0f * k) + k * (L.dot[i] - 1.0f));
    g[8 + i] = -scale * dlk;
    float const c = r * k / L.len[i];
    for (int a = 0; a < 3; ++a) g[16 + 3 * i + a] = -scale * c * (w[a] - L.dot[i] * L.mu[i][a]);
  }
}

// ------------------------------------------------------------- kernels
__device__ void load_weights(GuideSmem &S, const GuideDev &G) {
  const uint4 *src = reinterpret_cast<const uint4 *>(G.wblk);
  uint4 *dst = reinterpret_cast<uint4 *>(S.w);
  for (int i = threadIdx.x; i < static_cast<int>(kWBlkBytes / 16); i += blockDim.x) dst[i] = src[i];
  for (int i = threadIdx.x; i < kLayers * kW; i += blockDim.x) {
    int const l = i / kW, j = i % kW;
    S.bias[l][j] = G.params[param_b(l) + j];
  }
}

__device__ bool setup(GuideSmem &S, uint32_t ncols) {
  if (threadIdx.x == 0) {
    tc::mbar_init(tc::smem_addr(&S.mbar), 1);
    S.abort = 0;
  }
  if (threadIdx.x < 32) tc::tmem_alloc(&S.tmem, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  return true;
}

// Frees TMEM.  After a timed-out wait, first gives the MMAs still in flight
// one more bounded wait.
__device__ void teardown(GuideSmem &S, uint32_t ncols, bool aborted, uint32_t phase) {
  if (aborted) tc::mbar_wait(tc::smem_addr(&S.mbar), phase, kWaitLimit);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x < 32) tc::tmem_free(S.tmem, ncols);
}

// Raw outputs of n points (features: n x 6 = position, normal).
__global__ void __launch_bounds__(kGuideThreads, 1)
    k_guide_forward(GuideDev G, const float *__restrict__ feat, int n, float *__restrict__ out) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  GuideSmem &S = *reinterpret_cast<GuideSmem *>(smem_raw);
  load_weights(S, G);
  setup(S, 64);
  uint32_t phase = 0;
  bool aborted = false;
  int const ntiles = (n + kRows - 1) / kRows;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int const row = tile * kRows + threadIdx.x;
    float f[6] = {0, 0, 0, 0, 0, 1};
    if (row < n)
      for (int k = 0; k < 6; ++k) f[k] = feat[6 * static_cast<int64_t>(row) + k];
    encode_row(S, G, threadIdx.x, f);
    float o[kW];
    if (!forward_tile(S, phase, false, o)) {
      if (threadIdx.x == 0) atomicExch(G.err, 1);
      aborted = true;
      break;
    }
    if (row < n)
      for (int j = 0; j < kW; ++j) out[kW * static_cast<int64_t>(row) + j] = o[j];
  }
  teardown(S, 64, aborted, phase);
}

// Gradient of sum over records of -w * log p(dir) * scale, added to grad
// (flat parameter layout).  records: n x 10 = position, normal, direction, w.
__global__ void __launch_bounds__(kGuideThreads, 1)
    k_guide_gradient(GuideDev G, const float *__restrict__ rec, int n, float scale, float *__restrict__ grad) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  GuideSmem &S = *reinterpret_cast<GuideSmem *>(smem_raw);
  load_weights(S, G);
  for (int i = threadIdx.x; i < kLayers * kW; i += blockDim.x) (&S.db[0][0])[i] = 0.0f;
  setup(S, 512);
  uint32_t phase = 0;
  int const r = threadIdx.x;
  int const ntiles = (n + kRows - 1) / kRows;
  bool first = true, ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    int const row = tile * kRows + r;
    float f[6] = {0, 0, 0, 0, 0, 1}, dir[3] = {0, 0, 1}, wgt = 0.0f;
    if (row < n) {
      const float *q = rec + 10 * static_cast<int64_t>(row);
      for (int k = 0; k < 6; ++k) f[k] = q[k];
      dir[0] = q[6];
      dir[1] = q[7];
      dir[2] = q[8];
      wgt = q[9];
    }
    encode_row(S, G, r, f);
    float o[kW];
    if (!forward_tile(S, phase, true, o)) {
      ok = false;
      break;
    }
    // output deltas
    float g[kW];
    if (wgt != 0.0f && isfinite(wgt))
      loss_grad(o, dir, wgt * scale, g);
    else
      for (int j = 0; j < kW; ++j) g[j] = 0.0f;
#pragma unroll
    for (int c = 0; c < kW; c += 8) store_row8(S.d[0], r, c, kW, g + c);
    // backward: layer l's delta is in S.d[db_i]
    int dbuf = 0;
    for (int l = kLayers - 1; l >= 0 && ok; --l) {
      publish();
      if (r < kW) {  // bias gradient: column sums of the (bf16) delta
        float acc = 0.0f;
        for (int m = 0; m < kRows; ++m)
          acc += __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(S.d[dbuf] + tc::blocked_offset(m, r, kW)));
        S.db[l][r] += acc;
      }
      const uint8_t *act = l == 0 ? S.x : S.h[l - 1];
      int const K = layer_in(l);
      if (threadIdx.x == 0) {
        tc::fence_after_sync();
        uint32_t const da = tc::smem_addr(S.d[dbuf]), aa = tc::smem_addr(act);
        // dW_l^T (64 x K) += delta^T (64 x 128 rows) * act (128 rows x K)
        uint32_t const idw = tc::idesc_bf16(64, K, true, true);
        for (int ks = 0; ks < kRows / 16; ++ks)
          tc::mma_bf16(S.tmem + dw_col(l), tc::desc_mnmajor(da + ks * 2 * (kW / 8) * 128, kW),
                       tc::desc_mnmajor(aa + ks * 2 * (K / 8) * 128, K), idw, !first || ks > 0);
        if (l > 0) {
          // delta_{l-1} (128 x 64) = delta (128 x 64) * W_l (64 x 64, from W_l^T as MN-major)
          uint32_t const wb = tc::smem_addr(S.w) + wblk_off(l);
          uint32_t const idd = tc::idesc_bf16(kRows, kW, false, true);
          for (int ks = 0; ks < kW / 16; ++ks)
            tc::mma_bf16(S.tmem, tc::desc_kmajor(da + ks * 256, kW),
                         tc::desc_mnmajor(wb + ks * 2 * (K / 8) * 128, K), idd, ks > 0);
        }
        tc::mma_commit(tc::smem_addr(&S.mbar));
      }
      if (!await_mma(S, phase)) {
        ok = false;
        break;
      }
      if (l > 0) {
        float v[kW];
        read_acc(S, v);
        const uint8_t *hrow = S.h[l - 1];
#pragma unroll
        for (int c = 0; c < kW; c += 8) {
          uint4 const q = *reinterpret_cast<const uint4 *>(hrow + tc::blocked_offset(r, c, kW));
          uint32_t const hw[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            uint16_t const bits = static_cast<uint16_t>(hw[t >> 1] >> (16 * (t & 1)));
            if ((bits & 0x7FFFu) == 0u || (bits & 0x8000u)) v[c + t] = 0.0f;  // ReLU'(z) = [h > 0]
          }
        }
        dbuf ^= 1;
#pragma unroll
        for (int c = 0; c < kW; c += 8) store_row8(S.d[dbuf], r, c, kW, v + c);
      }
    }
    first = false;
  }
  if (!ok && threadIdx.x == 0) atomicExch(G.err, 1);
  // weight gradients out of TMEM (M = 64 layout) and bias gradients
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (ok && !first) {
    int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t const lane_base = static_cast<uint32_t>(warp * 32) << 16;
    int const nrow = warp * 16 + lane;  // output unit of this lane (lanes < 16)
    for (int l = 0; l < kLayers; ++l) {
      int const K = layer_in(l);
      for (int c = 0; c < K; c += 16) {
        float v[16];
        tc::tmem_ld16(S.tmem + lane_base + dw_col(l) + c, v);
        tc::tmem_wait_ld();
        if (lane < 16)
          for (int t = 0; t < 16; ++t) atomicAdd(&grad[param_w(l) + (c + t) * kW + nrow], v[t]);
      }
    }
    for (int i = threadIdx.x; i < kLayers * kW; i += blockDim.x)
      atomicAdd(&grad[param_b(i / kW) + i % kW], (&S.db[0][0])[i]);
  }
  teardown(S, 512, !ok, phase);
}

// fp32 master weights -> blocked bf16 W^T per layer.
__global__ void k_guide_pack(const float *__restrict__ params, uint8_t *__restrict__ wblk) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  int l = 0, rem = i;
  while (l < kLayers && rem >= layer_in(l) * kW) {
    rem -= layer_in(l) * kW;
    ++l;
  }
  if (l >= kLayers) return;
  int const K = layer_in(l);
  int const k = rem / kW, nn = rem % kW;  // W_l[k][nn]
  __nv_bfloat16 const b = __float2bfloat16_rn(params[param_w(l) + k * kW + nn]);
  *reinterpret_cast<__nv_bfloat16 *>(wblk + wblk_off(l) + tc::blocked_offset(nn, k, K)) = b;
}

__global__ void k_guide_adam(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m,
                             float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  float const gi = g[i];
  float const mi = b1 * m[i] + (1.0f - b1) * gi;
  float const vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  g[i] = 0.0f;
}

}  // namespace

// ---------------------------------------------------------------- host
struct GuideImpl {
  int device = 0;
  xyzgpu_guide_config cfg{};
  SceneImpl *scene = nullptr;
  float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
  uint8_t *d_wblk = nullptr;
  int *d_err = nullptr;
  int64_t step = 0;
  float lo[3] = {0, 0, 0}, inv_ext[3] = {1, 1, 1};
};

namespace {

GuideDev guide_dev(const GuideImpl &g) {
  GuideDev d;
  d.wblk = g.d_wblk;
  d.params = g.d_params;
  for (int k = 0; k < 3; ++k) {
    d.lo[k] = g.lo[k];
    d.inv_ext[k] = g.inv_ext[k];
  }
  d.err = g.d_err;
  return d;
}

int pack(GuideImpl &g, cudaStream_t st) {
  int const nw = kParams - kLayers * kW;
  k_guide_pack<<<(nw + 255) / 256, 256, 0, st>>>(g.d_params, g.d_wblk);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int grid_for(int device, int n) {
  int const tiles = (n + kRows - 1) / kRows;
  return std::max(1, std::min(tiles, sm_count(device)));
}

// splitmix64 -> uniform in [-1, 1)
double rand_sym(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

int check_err(GuideImpl &g, cudaStream_t st, const char *who) {
  int e = 0;
  XYZ_CUDA_TRY(cudaMemcpyAsync(&e, g.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  if (e) return set_error(XYZGPU_E_CUDA, "%s: a tensor-core wait timed out", who);
  return XYZGPU_OK;
}

}  // namespace

int guide_forward_launch(GuideImpl &g, const float *feat, int n, float *out, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    XYZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(sizeof(GuideSmem))));
    attr = true;
  }
  if (n <= 0) return XYZGPU_OK;
  k_guide_forward<<<grid_for(g.device, n), kGuideThreads, sizeof(GuideSmem), st>>>(guide_dev(g), feat, n, out);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int guide_gradient_launch(GuideImpl &g, const float *rec, int n, float scale, float *grad, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    XYZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_gradient, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(sizeof(GuideSmem))));
    attr = true;
  }
  if (n <= 0) return XYZGPU_OK;
  k_guide_gradient<<<grid_for(g.device, n), kGuideThreads, sizeof(GuideSmem), st>>>(guide_dev(g), rec, n, scale,
                                                                                     grad);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int guide_adam_launch(GuideImpl &g, cudaStream_t st) {
  g.step += 1;
  float const b1 = 0.9f, b2 = 0.99f;
  float const c1 = static_cast<float>(1.0 - std::pow(0.9, static_cast<double>(g.step)));
  float const c2 = static_cast<float>(1.0 - std::pow(0.99, static_cast<double>(g.step)));
  k_guide_adam<<<(kParams + 255) / 256, 256, 0, st>>>(g.d_params, g.d_grad, g.d_m, g.d_v, g.cfg.learning_rate, b1,
                                                      b2, 1e-8f, c1, c2);
  XYZ_CUDA_TRY(cudaGetLastError());
  return pack(g, st);
}

}  // namespace xyzgpu

using namespace xyzgpu;

struct xyzgpu_guide_s {
  GuideImpl g;
};

extern "C" {

void xyzgpu_guide_config_default(xyzgpu_guide_config *c) {
  if (!c) return;
  c->alpha = 0.5f;
  c->learning_rate = 1e-3f;
  c->batch_size = 1 << 16;
  c->steps_per_pass = 16;
  c->train_bounces = 2;
  c->seed = 0;
}

void xyzgpu_guide_destroy(xyzgpu_guide h) {
  if (!h) return;
  GuideImpl &g = h->g;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(g.device);
  cudaDeviceSynchronize();
  cudaFree(g.d_params);
  cudaFree(g.d_grad);
  cudaFree(g.d_m);
  cudaFree(g.d_v);
  cudaFree(g.d_wblk);
  cudaFree(g.d_err);
  cudaSetDevice(prev);
  delete h;
}

int xyzgpu_guide_create(xyzgpu_scene scene, const xyzgpu_guide_config *cfg, xyzgpu_guide *out) {
  clear_error();
  if (!scene || !out) return set_error(XYZGPU_E_INVALID, "guide_create: null argument");
  *out = nullptr;
  xyzgpu_guide_config c;
  if (cfg)
    c = *cfg;
  else
    xyzgpu_guide_config_default(&c);
  if (!(c.alpha >= 0.0f && c.alpha < 1.0f) || !(c.learning_rate > 0.0f) || c.batch_size < 1 ||
      c.steps_per_pass < 0 || c.train_bounces < 0 || c.train_bounces > 8)
    return set_error(XYZGPU_E_INVALID, "guide_create: configuration out of range");
  auto *h = new (std::nothrow) xyzgpu_guide_s();
  if (!h) return set_error(XYZGPU_E_NOMEM, "guide_create: host allocation failed");
  GuideImpl &g = h->g;
  SceneImpl *s = reinterpret_cast<SceneImpl *>(scene);
  g.scene = s;
  g.device = s->device;
  g.cfg = c;
  float const lo[3] = {s->dev.bmin.x, s->dev.bmin.y, s->dev.bmin.z};
  float const hi[3] = {s->dev.bmax.x, s->dev.bmax.y, s->dev.bmax.z};
  for (int k = 0; k < 3; ++k) {
    g.lo[k] = lo[k];
    float const ext = hi[k] - lo[k];
    g.inv_ext[k] = ext > 0.0f ? 1.0f / ext : 1.0f;
  }
  auto fail = [&](int rc) {
    xyzgpu_guide_destroy(h);
    return rc;
  };
  if (cudaSetDevice(g.device) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_params), kParams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_grad), kParams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_m), kParams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_v), kParams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_wblk), kWBlkBytes) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_err), sizeof(int)) != cudaSuccess)
    return fail(set_error(XYZGPU_E_NOMEM, "guide_create: device allocation failed"));
  // He-uniform hidden layers, a small output layer (near-uniform mixture at
  // the start), zero biases
  std::vector<float> p(kParams, 0.0f);
  uint64_t st = c.seed * 0x2545F4914F6CDD1Dull + 1;
  for (int l = 0; l < kLayers; ++l) {
    double const bound = std::sqrt(6.0 / layer_in(l)) * (l == kLayers - 1 ? 0.1 : 1.0);
    for (int i = 0; i < layer_in(l) * kW; ++i) p[param_w(l) + i] = static_cast<float>(bound * rand_sym(st));
  }
  if (cudaMemcpy(g.d_params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(g.d_grad, 0, kParams * sizeof(float)) != cudaSuccess ||
      cudaMemset(g.d_m, 0, kParams * sizeof(float)) != cudaSuccess ||
      cudaMemset(g.d_v, 0, kParams * sizeof(float)) != cudaSuccess ||
      cudaMemset(g.d_err, 0, sizeof(int)) != cudaSuccess)
    return fail(set_error(XYZGPU_E_CUDA, "guide_create: initialisation failed"));
  int rc = pack(g, nullptr);
  if (rc) return fail(rc);
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) return fail(set_error(XYZGPU_E_CUDA, "guide_create: pack failed"));
  *out = h;
  return XYZGPU_OK;
}

int xyzgpu_guide_get_params(xyzgpu_guide h, float *params) {
  clear_error();
  if (!h || !params) return set_error(XYZGPU_E_INVALID, "guide_get_params: null argument");
  XYZ_CUDA_TRY(cudaSetDevice(h->g.device));
  XYZ_CUDA_TRY(cudaMemcpy(params, h->g.d_params, kParams * sizeof(float), cudaMemcpyDeviceToHost));
  return XYZGPU_OK;
}

int xyzgpu_guide_set_params(xyzgpu_guide h, const float *params) {
  clear_error();
  if (!h || !params) return set_error(XYZGPU_E_INVALID, "guide_set_params: null argument");
  GuideImpl &g = h->g;
  for (int i = 0; i < kParams; ++i)
    if (!std::isfinite(params[i])) return set_error(XYZGPU_E_INVALID, "guide_set_params: parameter %d is not finite", i);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  XYZ_CUDA_TRY(cudaMemcpy(g.d_params, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
  XYZ_CUDA_TRY(cudaMemset(g.d_m, 0, kParams * sizeof(float)));
  XYZ_CUDA_TRY(cudaMemset(g.d_v, 0, kParams * sizeof(float)));
  g.step = 0;
  int const rc = pack(g, nullptr);
  if (rc) return rc;
  XYZ_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return XYZGPU_OK;
}

int xyzgpu_guide_forward(xyzgpu_guide h, const float *features, int n, float *out, void *stream) {
  clear_error();
  if (!h || n < 0 || (n > 0 && (!features || !out))) return set_error(XYZGPU_E_INVALID, "guide_forward: bad argument");
  GuideImpl &g = h->g;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  XYZ_CUDA_TRY(cudaMemsetAsync(g.d_err, 0, sizeof(int), st));
  int const rc = guide_forward_launch(g, features, n, out, st);
  if (rc) return rc;
  return check_err(g, st, "guide_forward");
}

int xyzgpu_guide_gradient(xyzgpu_guide h, const float *records, int n, float scale, float *grad, void *stream) {
  clear_error();
  if (!h || n < 0 || (n > 0 && (!records || !grad)) || !std::isfinite(scale))
    return set_error(XYZGPU_E_INVALID, "guide_gradient: bad argument");
  GuideImpl &g = h->g;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  XYZ_CUDA_TRY(cudaMemsetAsync(g.d_err, 0, sizeof(int), st));
  int const rc = guide_gradient_launch(g, records, n, scale, grad, st);
  if (rc) return rc;
  return check_err(g, st, "guide_gradient");
}

int xyzgpu_guide_train_step(xyzgpu_guide h, const float *records, int n, void *stream) {
  clear_error();
  if (!h || n <= 0 || !records) return set_error(XYZGPU_E_INVALID, "guide_train_step: bad argument");
  GuideImpl &g = h->g;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  XYZ_CUDA_TRY(cudaMemsetAsync(g.d_err, 0, sizeof(int), st));
  int rc = guide_gradient_launch(g, records, n, 1.0f / static_cast<float>(n), g.d_grad, st);
  if (rc) return rc;
  rc = guide_adam_launch(g, st);
  if (rc) return rc;
  return check_err(g, st, "guide_train_step");
}

}  // extern "C"
