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
// memory and the accumulator in TMEM; the epilogue (ReLU, bf16 pack) reads
// the accumulator back with tcgen05.ld, one TMEM lane per thread = one
// row.  The bias enters the accumulator as one more MMA (K = 16) of a
// constant tile of ones with the bias split into three bf16 parts (hi, mid,
// lo: their sum is the fp32 bias to within fp32 rounding), so the epilogue is
// only ReLU and the bf16 pack, one cvt.rn.relu.bf16x2 per pair.  Training runs the forward pass, the loss gradient at the output, and
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
#include <cuda_fp16.h>

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
constexpr int kHBytes = kRows * kW * 2;  // one hidden activation buffer
constexpr int kBiasK = 16;               // K of the bias MMA (columns 0..2 used)

// The weights as the tensor cores read them: blocked bf16 W^T per layer, the
// ones tile (128 x 16, columns 0..2 = 1) and per layer the bias tile (64 x 16,
// columns 0..2 = the bias's hi, mid and lo bf16 parts).
struct WeightsSmem {
  uint8_t w[kWBlkBytes];
  uint8_t ones[kRows * kBiasK * 2];
  uint8_t bias[kLayers][kW * kBiasK * 2];
};
// The same image lives in global memory (GuideImpl::d_wblk), rebuilt by
// k_guide_pack after every weight update; each CTA copies it as is.
constexpr uint32_t kOnesOff = kWBlkBytes;
constexpr uint32_t kBiasOff = kOnesOff + kRows * kBiasK * 2;
constexpr uint32_t kWImageBytes = kBiasOff + kLayers * kW * kBiasK * 2;  // 71680
static_assert(sizeof(WeightsSmem) == kWImageBytes && kWImageBytes % 16 == 0, "weight image layout");

// TMEM columns: [0, 64) the working accumulator; weight gradients (M = 64
// layout: rows 16w..16w+15 in lanes 32w..32w+15) of layer 0 at [64, 256),
// layers 1..4 at 256 + 64 (l - 1).
__device__ __forceinline__ uint32_t dw_col(int l) { return l == 0 ? 64u : 256u + 64u * (l - 1); }

struct __align__(128) GuideSmem {
  WeightsSmem wt;
  uint8_t x[kRows * kIn * 2];
  uint8_t h[4][kRows * kW * 2];
  uint8_t d[2][kRows * kW * 2];
  float db[kLayers][kW];
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};

struct GuideDev {
  const uint8_t *wblk;  // packed weight image (WeightsSmem layout)
  const float *params;  // fp32 master (biases read from here)
  float lo[3], inv_ext[3];  // position normalisation: s = (p - lo) * inv_ext
  int *err;
};

// ---------------------------------------------------------------- encoding
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 const v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// ReLU and bf16 pack of two values (a in the low half).
__device__ __forceinline__ uint32_t pack_relu_bf16x2(float a, float b) {
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
  return d;
}

__device__ __forceinline__ void store_row8_relu(uint8_t *buf, int r, int c, int cols, const float *v) {
  uint4 q;
  q.x = pack_relu_bf16x2(v[0], v[1]);
  q.y = pack_relu_bf16x2(v[2], v[3]);
  q.z = pack_relu_bf16x2(v[4], v[5]);
  q.w = pack_relu_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(buf + tc::blocked_offset(r, c, cols)) = q;
}

__device__ __forceinline__ void store_row8(uint8_t *buf, int r, int c, int cols, const float *v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(buf + tc::blocked_offset(r, c, cols)) = q;
}

// Row r of the input encoding from a raw point (position, normal): per
// input s in [0, 1], 32 bins of exp(-(s - (j + 1/2) / 32)^2 / (2 sigma^2)),
// sigma = 1/32.  Bins more than 4.5 sigma from s are exactly 0 (exp(-10) and
// below; the oracle applies the same cut): an input's 32 columns are cleared,
// then the at most 10 bins of its window are computed.  In bin units (u = 32 s,
// t_j = u - j - 1/2) the bins are g_j = exp(-t_j^2 / 2), and
// g_{j+1} = g_j exp(t_j - 1/2), exp(t_{j+1} - 1/2) = exp(t_j - 1/2) / e: two
// exponentials per input and two products per bin, from the even column at
// or below the window's first bin.  The window is stored as bf16 pairs at
// even columns (4-byte stores, a neighbour outside the window being 0),
// which halves the shared-memory stores of one-by-one 2-byte writes.
//
// Input coordinate of feature `dim` in [0, 1]: the position in the scene's
// bounds, a normal component mapped from [-1, 1].
__device__ __forceinline__ float encode_coord(const GuideDev &G, int dim, float f) {
  float const s = dim < 3 ? (f - G.lo[dim]) * G.inv_ext[dim] : (f + 1.0f) * 0.5f;
  return fminf(fmaxf(s, 0.0f), 1.0f);
}

// The kBins columns c0 .. c0 + kBins - 1 of row r of a blocked buffer of C
// columns: one input coordinate s.
__device__ __forceinline__ void encode_dim(uint8_t *x, int r, int C, int c0, float s) {
#pragma unroll
  for (int q = 0; q < kBins; q += 8)
    *reinterpret_cast<uint4 *>(x + tc::blocked_offset(r, c0 + q, C)) = make_uint4(0, 0, 0, 0);
  float const u = s * static_cast<float>(kBins);
  // the even column at or below the first bin within 4.5 sigma: the at most
  // 10 bins within reach lie in the 12 columns from it, stored as 6 pairs
  int const e0 = max(0, static_cast<int>(ceilf(u - 5.0f))) & ~1;
  float const t0 = u - (static_cast<float>(e0) + 0.5f);
  float g = __expf(-0.5f * t0 * t0);
  float ratio = __expf(t0 - 0.5f);
  float v[12];
#pragma unroll
  for (int t = 0; t < 12; ++t) {
    v[t] = (e0 + t < kBins && fabsf(t0 - static_cast<float>(t)) <= 4.5f) ? g : 0.0f;
    g *= ratio;
    ratio *= 0.36787944117144233f;  // 1 / e
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int const c = e0 + 2 * k;
    if (c < kBins) {
      __nv_bfloat162 const pr = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
      *reinterpret_cast<__nv_bfloat162 *>(x + tc::blocked_offset(r, c0 + c, C)) = pr;
    }
  }
}

__device__ void encode_row(uint8_t *x, int r, const GuideDev &G, const float f[6]) {
#pragma unroll
  for (int dim = 0; dim < 6; ++dim) encode_dim(x, r, kIn, dim * kBins, encode_coord(G, dim, f[dim]));
}

// ---------------------------------------------------------------- tiles
// The 128 rows one group of four warps works on: its buffers, its TMEM
// accumulator (64 columns), its completion mbarrier and its barrier (0 = the
// whole CTA, else a named barrier of the group's 128 threads).
struct Tile {
  uint8_t *x;     // encoding [128][192]
  uint8_t *h;     // hidden outputs [128][64] at h + l * kHBytes: all four kept for training,
                  // else two buffers alternate (l & 1)
  uint32_t tmem;
  uint32_t mbar;
  int bar;
  int t;          // this thread's row
};

__device__ __forceinline__ void tile_sync(int bar) {
  if (bar == 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, 128;" ::"r"(bar) : "memory");
}

// Uniform over the group: true if any thread's flag is set.
__device__ __forceinline__ bool tile_any(int bar, bool flag) {
  if (bar == 0) return __syncthreads_or(flag ? 1 : 0) != 0;
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"(flag ? 1u : 0u), "r"(bar)
      : "memory");
  return r != 0;
}

// Shared-memory writes of the group become visible to the tensor cores.
__device__ __forceinline__ void publish(int bar) {
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  tile_sync(bar);
}

// Waits for the group's committed MMAs; false (uniformly) if any thread gave
// up, in which case `phase` still names the pending completion.
__device__ __forceinline__ bool await_mma(const Tile &c, uint32_t &phase) {
  bool const ok = tc::mbar_wait(c.mbar, phase, kWaitLimit);
  tc::fence_after_sync();
  if (tile_any(c.bar, !ok)) return false;
  phase ^= 1u;
  return true;
}

__device__ __forceinline__ void issue_forward(const WeightsSmem &wt, int l, const uint8_t *in, uint32_t tmem) {
  int const K = layer_in(l);
  uint32_t const a0 = tc::smem_addr(in), b0 = tc::smem_addr(wt.w) + wblk_off(l);
  uint32_t const id = tc::idesc_bf16(kRows, kW, false, false);
  // D = ones * bias_parts^T (every row the bias), then D += in * W
  tc::mma_bf16(tmem, tc::desc_kmajor(tc::smem_addr(wt.ones), kBiasK), tc::desc_kmajor(tc::smem_addr(wt.bias[l]), kBiasK),
               id, false);
  for (int ks = 0; ks < K / 16; ++ks)
    tc::mma_bf16(tmem, tc::desc_kmajor(a0 + ks * 256, K), tc::desc_kmajor(b0 + ks * 256, K), id, true);
}

// This thread's row of an accumulator (64 fp32); a warp reads the 32 TMEM
// lanes of its quarter (32 * (warp % 4)).
__device__ __forceinline__ void read_acc(uint32_t tmem, float *v) {
  uint32_t const taddr = tmem + (((threadIdx.x >> 5) & 3u) << 21);
#pragma unroll
  for (int c = 0; c < kW; c += 16) tc::tmem_ld16(taddr + c, v + c);
  tc::tmem_wait_ld();
}

// Forward pass of the tile whose encoding is in c.x; leaves this thread's row
// of raw outputs (with bias) in out[64].
__device__ bool forward(const WeightsSmem &wt, Tile &c, uint32_t &phase, bool keep, float *out) {
  const uint8_t *in = c.x;
  for (int l = 0; l < kLayers; ++l) {
    publish(c.bar);
    if (c.t == 0) {
      tc::fence_after_sync();
      issue_forward(wt, l, in, c.tmem);
      tc::mma_commit(c.mbar);
    }
    if (!await_mma(c, phase)) return false;
    float v[kW];
    read_acc(c.tmem, v);
    if (l == kLayers - 1) {
#pragma unroll
      for (int j = 0; j < kW; ++j) out[j] = v[j];
      break;
    }
    uint8_t *dst = c.h + (keep ? l : (l & 1)) * kHBytes;
#pragma unroll
    for (int q = 0; q < kW; q += 8) store_row8_relu(dst, c.t, q, kW, v + q);
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

// ------------------------------------------------------------- training state
// Device-resident training state, so that a whole training pass (records ->
// steps_per_pass x (gradient, Adam) -> bookkeeping) runs without the host
// reading anything back and can be replayed as one CUDA graph.
struct TrainState {
  long long step;               // Adam steps taken
  long long offset;             // rolling start of the next batch in the training rows
  unsigned long long trained;   // training rows produced so far
  int count;                    // rows k_guide_records wrote (may exceed the buffer)
  int pad;
};

// Rows of one gradient launch: explicit (rec, n, scale), or - with ts set -
// batch `step_rel` of a training pass over min(ts->count, cap) rows at rec:
// bs = min(batch, rows) rows from (ts->offset + step_rel * bs) mod rows,
// moved back to rows - bs if they would run past the end, scale 1 / bs.
struct GradArgs {
  const float *rec;
  int n;
  float scale;
  float *grad;
  const TrainState *ts;
  long long cap;
  int step_rel;
  int batch;
};

__device__ __forceinline__ bool grad_rows(const GradArgs &A, const float *&rec, int &n, float &scale) {
  rec = A.rec;
  n = A.n;
  scale = A.scale;
  if (!A.ts) return n > 0;
  long long const rows = min(static_cast<long long>(A.ts->count), A.cap);
  if (rows <= 0) return false;
  long long const bs = min(static_cast<long long>(A.batch), rows);
  long long off = (A.ts->offset + static_cast<long long>(A.step_rel) * bs) % rows;
  if (off + bs > rows) off = rows - bs;
  rec += 10 * off;
  n = static_cast<int>(bs);
  scale = 1.0f / static_cast<float>(bs);
  return true;
}

// ------------------------------------------------------------- kernels
// Copies the packed weight image (weights, ones tile, bias tiles) into shared
// memory: 4,480 independent 16-byte loads, several in flight per thread.
__device__ void load_weights(WeightsSmem &wt, const GuideDev &G) {
  const uint4 *src = reinterpret_cast<const uint4 *>(G.wblk);
  uint4 *dst = reinterpret_cast<uint4 *>(&wt);
#pragma unroll 4
  for (int i = threadIdx.x; i < static_cast<int>(kWImageBytes / 16); i += blockDim.x) dst[i] = __ldg(&src[i]);
}

// mbarriers (count 1) and `ncols` TMEM columns for the CTA.
__device__ void setup(uint64_t *mbar, int nbar, uint32_t *tmem_slot, uint32_t ncols) {
  if (threadIdx.x == 0)
    for (int i = 0; i < nbar; ++i) tc::mbar_init(tc::smem_addr(&mbar[i]), 1);
  if (threadIdx.x < 32) tc::tmem_alloc(tmem_slot, ncols);
  tc::fence_smem_to_async();  // the weights every thread stored, for every group's MMAs
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// Frees TMEM.  A group whose wait timed out first gives its MMAs still in
// flight one more bounded wait.
__device__ void teardown(uint32_t tmem, uint32_t ncols, bool aborted, uint32_t mbar, uint32_t phase) {
  if (aborted) tc::mbar_wait(mbar, phase, kWaitLimit);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x < 32) tc::tmem_free(tmem, ncols);
}

// Inference CTAs: four groups of four warps, each with its own 128-row tile,
// two 16 KB buffers and accumulator, sharing the weights; while one group waits
// for its MMAs the others run their encodings, epilogues or gathers.  The first
// layer runs in three K-chunks of two inputs (64 columns) through the two
// buffers, the hidden activations then alternate between them
// (forward_infer).
constexpr int kGroups = 4;
constexpr int kInferThreads = kGroups * kRows;

struct __align__(128) InferSmem {
  WeightsSmem wt;
  uint8_t x[kGroups][2 * kHBytes];
  uint64_t mbar[kGroups];
  uint32_t tmem;
};

static_assert(sizeof(InferSmem) <= 227 * 1024, "inference CTA shared memory");
static_assert(sizeof(GuideSmem) <= 227 * 1024, "training CTA shared memory");

__device__ Tile infer_tile(InferSmem &S, int gi) {
  Tile c;
  c.x = S.x[gi];
  c.h = S.x[gi];
  c.tmem = S.tmem + 64u * static_cast<uint32_t>(gi);
  c.mbar = tc::smem_addr(&S.mbar[gi]);
  c.bar = 1 + gi;
  c.t = threadIdx.x & (kRows - 1);
  return c;
}

// Forward pass of this thread's row from its features (inference CTAs),
// leaving the raw outputs (with bias) in out[64].  The first layer's K-chunks
// go through the group's buffers A and B: chunk 0 (inputs 0, 1) -> A, chunk 1
// -> B, and chunk 2 -> A once chunk 0's MMAs (committed on their own) have
// read it, so a chunk's MMAs overlap the next chunk's encoding.  Hidden layer
// l - 1's activations go to A for even l - 1, B for odd: the MMA that read that
// buffer last has completed by then.
__device__ bool forward_infer(const WeightsSmem &wt, const GuideDev &G, Tile &c, uint32_t &phase,
                              const float f[6], float *out) {
  uint8_t *const buf[2] = {c.x, c.x + kHBytes};
  constexpr int kChunk = 2 * kBins;  // columns of a K-chunk
  uint32_t const id = tc::idesc_bf16(kRows, kW, false, false);
  uint32_t const b0 = tc::smem_addr(wt.w) + wblk_off(0);
#pragma unroll
  for (int k = 0; k < kIn / kChunk; ++k) {
    uint8_t *const dst = buf[k & 1];
    if (k == 2 && !await_mma(c, phase)) return false;
    encode_dim(dst, c.t, kChunk, 0, encode_coord(G, 2 * k, f[2 * k]));
    encode_dim(dst, c.t, kChunk, kBins, encode_coord(G, 2 * k + 1, f[2 * k + 1]));
    publish(c.bar);
    if (c.t == 0) {
      tc::fence_after_sync();
      if (k == 0)
        tc::mma_bf16(c.tmem, tc::desc_kmajor(tc::smem_addr(wt.ones), kBiasK),
                     tc::desc_kmajor(tc::smem_addr(wt.bias[0]), kBiasK), id, false);
      uint32_t const a0 = tc::smem_addr(dst);
#pragma unroll
      for (int ks = 0; ks < kChunk / 16; ++ks)
        tc::mma_bf16(c.tmem, tc::desc_kmajor(a0 + ks * 256, kChunk),
                     tc::desc_kmajor(b0 + (k * (kChunk / 16) + ks) * 256, kIn), id, true);
      if (k != 1) tc::mma_commit(c.mbar);
    }
  }
  if (!await_mma(c, phase)) return false;
  float v[kW];
  read_acc(c.tmem, v);
  for (int l = 1; l < kLayers; ++l) {
    uint8_t *const dst = buf[(l - 1) & 1];
#pragma unroll
    for (int q = 0; q < kW; q += 8) store_row8_relu(dst, c.t, q, kW, v + q);
    publish(c.bar);
    if (c.t == 0) {
      tc::fence_after_sync();
      issue_forward(wt, l, dst, c.tmem);
      tc::mma_commit(c.mbar);
    }
    if (!await_mma(c, phase)) return false;
    read_acc(c.tmem, v);
  }
#pragma unroll
  for (int j = 0; j < kW; ++j) out[j] = v[j];
  return true;
}

// Raw outputs of n points (features: n x 6 = position, normal).
__global__ void __launch_bounds__(kInferThreads, 1)
    k_guide_forward(const __grid_constant__ GuideDev G, const float *__restrict__ feat, int n, float *__restrict__ out) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  InferSmem &S = *reinterpret_cast<InferSmem *>(smem_raw);
  load_weights(S.wt, G);
  setup(S.mbar, kGroups, &S.tmem, 256);
  int const gi = threadIdx.x >> 7;
  Tile c = infer_tile(S, gi);
  uint32_t phase = 0;
  bool aborted = false;
  int const ntiles = (n + kRows - 1) / kRows;
  for (int tile = kGroups * blockIdx.x + gi; tile < ntiles; tile += kGroups * gridDim.x) {
    int const row = tile * kRows + c.t;
    float f[6] = {0, 0, 0, 0, 0, 1};
    if (row < n)
      for (int k = 0; k < 6; ++k) f[k] = feat[6 * static_cast<int64_t>(row) + k];
    float o[kW];
    if (!forward_infer(S.wt, G, c, phase, f, o)) {
      if (c.t == 0) atomicExch(G.err, 1);
      aborted = true;
      break;
    }
    if (row < n)
      for (int j = 0; j < kW; ++j) out[kW * static_cast<int64_t>(row) + j] = o[j];
  }
  teardown(S.tmem, 256, aborted, c.mbar, phase);
}

// Gradient of sum over records of -w * log p(dir) * scale, added to grad
// (flat parameter layout).  records: n x 10 = position, normal, direction, w.
__global__ void __launch_bounds__(kGuideThreads, 1)
    k_guide_gradient(const __grid_constant__ GuideDev G, const __grid_constant__ GradArgs A) {
  const float *rec;
  int n;
  float scale;
  if (!grad_rows(A, rec, n, scale)) return;  // uniform over the grid: no rows
  float *__restrict__ grad = A.grad;
  extern __shared__ __align__(128) uint8_t smem_raw[];
  GuideSmem &S = *reinterpret_cast<GuideSmem *>(smem_raw);
  load_weights(S.wt, G);
  for (int i = threadIdx.x; i < kLayers * kW; i += blockDim.x) (&S.db[0][0])[i] = 0.0f;
  setup(&S.mbar, 1, &S.tmem, 512);
  Tile c;
  c.x = S.x;
  c.h = S.h[0];
  c.tmem = S.tmem;
  c.mbar = tc::smem_addr(&S.mbar);
  c.bar = 0;
  c.t = threadIdx.x;
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
    encode_row(S.x, r, G, f);
    float o[kW];
    if (!forward(S.wt, c, phase, true, o)) {
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
    for (int q = 0; q < kW; q += 8) store_row8(S.d[0], r, q, kW, g + q);
    // backward: layer l's delta is in S.d[dbuf]
    int dbuf = 0;
    for (int l = kLayers - 1; l >= 0 && ok; --l) {
      publish(0);
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
          uint32_t const wb = tc::smem_addr(S.wt.w) + wblk_off(l);
          uint32_t const idd = tc::idesc_bf16(kRows, kW, false, true);
          for (int ks = 0; ks < kW / 16; ++ks)
            tc::mma_bf16(S.tmem, tc::desc_kmajor(da + ks * 256, kW),
                         tc::desc_mnmajor(wb + ks * 2 * (K / 8) * 128, K), idd, ks > 0);
        }
        tc::mma_commit(c.mbar);
      }
      if (!await_mma(c, phase)) {
        ok = false;
        break;
      }
      if (l > 0) {
        float v[kW];
        read_acc(S.tmem, v);
        const uint8_t *hrow = S.h[l - 1];
#pragma unroll
        for (int q = 0; q < kW; q += 8) {
          uint4 const hq = *reinterpret_cast<const uint4 *>(hrow + tc::blocked_offset(r, q, kW));
          uint32_t const hw[4] = {hq.x, hq.y, hq.z, hq.w};
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            uint16_t const bits = static_cast<uint16_t>(hw[t >> 1] >> (16 * (t & 1)));
            if ((bits & 0x7FFFu) == 0u || (bits & 0x8000u)) v[q + t] = 0.0f;  // ReLU'(z) = [h > 0]
          }
        }
        dbuf ^= 1;
#pragma unroll
        for (int q = 0; q < kW; q += 8) store_row8(S.d[dbuf], r, q, kW, v + q);
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
      for (int q = 0; q < K; q += 16) {
        float v[16];
        tc::tmem_ld16(S.tmem + lane_base + dw_col(l) + q, v);
        tc::tmem_wait_ld();
        if (lane < 16)
          for (int t = 0; t < 16; ++t) atomicAdd(&grad[param_w(l) + (q + t) * kW + nrow], v[t]);
      }
    }
    for (int i = threadIdx.x; i < kLayers * kW; i += blockDim.x)
      atomicAdd(&grad[param_b(i / kW) + i % kW], (&S.db[0][0])[i]);
  }
  teardown(S.tmem, 512, !ok, c.mbar, phase);
}

// Guide inference for a render's extension queue: the hit point and shading
// normal of every queue entry (computed as the shading kernel does) through
// the network; per entry the mixture (weights, concentrations, means) as 40
// fp16 values.  Persistent CTAs of three groups; the queue length is read on
// the device.
struct InferArgs {
  const float4 *qo, *qd, *hits;
  const int32_t *count;
  const float4 *tri_ng, *tri_sn;
  __half *mix;
};

// One queue entry's inputs: hit record, ray origin and direction, and the
// hit triangle's shading normals (n0, n1 - n0, n2 - n0; or the geometric
// normal in n0 for scenes without normals).  The kernel loads them one and
// two tiles ahead so that these gathers overlap the network of the current
// tile.
struct InferRow {
  float4 h, o, d, n0, s1, s2;
};

__device__ __forceinline__ float4 miss_hit() { return make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1)); }

// Ray and normals of entry i (its hit record r.h already loaded).
__device__ __forceinline__ void infer_gather(const InferArgs &I, int i, InferRow &r) {
  int32_t const code = __float_as_int(r.h.w);
  if (code < 0) return;
  int const tri = code >> 1;
  r.o = I.qo[i];
  r.d = I.qd[i];
  if (I.tri_sn) {
    r.n0 = __ldg(&I.tri_sn[3 * tri]);
    r.s1 = __ldg(&I.tri_sn[3 * tri + 1]);
    r.s2 = __ldg(&I.tri_sn[3 * tri + 2]);
  } else {
    r.n0 = __ldg(&I.tri_ng[tri]);
  }
}

// Surface point (position, shading normal facing the incoming ray) of a
// gathered entry, as the shading kernel computes it; the default row for a
// miss.
__device__ void infer_features(const InferArgs &I, const InferRow &r, float f[6]) {
  f[0] = f[1] = f[2] = f[3] = f[4] = 0.0f;
  f[5] = 1.0f;
  int32_t const code = __float_as_int(r.h.w);
  if (code < 0) return;
  f3 const pos = add3(xyz3(r.o), scl3(xyz3(r.d), r.h.x));
  f3 sn;
  if (I.tri_sn) {
    sn = normalize3(add3(add3(xyz3(r.n0), scl3(xyz3(r.s1), r.h.y)), scl3(xyz3(r.s2), r.h.z)));
  } else {
    f3 const z = mk3(0.0f, 0.0f, 0.0f);
    sn = normalize3(add3(add3(xyz3(r.n0), scl3(z, r.h.y)), scl3(z, r.h.z)));
  }
  if (code & 1) sn = neg3(sn);
  f[0] = pos.x, f[1] = pos.y, f[2] = pos.z, f[3] = sn.x, f[4] = sn.y, f[5] = sn.z;
}

__global__ void __launch_bounds__(kInferThreads, 1) k_guide_infer(const __grid_constant__ GuideDev G, InferArgs I) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  InferSmem &S = *reinterpret_cast<InferSmem *>(smem_raw);
  load_weights(S.wt, G);
  setup(S.mbar, kGroups, &S.tmem, 256);
  int const gi = threadIdx.x >> 7;
  Tile c = infer_tile(S, gi);
  uint32_t phase = 0;
  bool aborted = false;
  int const n = *I.count;
  int const ntiles = (n + kRows - 1) / kRows;
  int const step = kGroups * gridDim.x;
  int tile = kGroups * blockIdx.x + gi;
  // this thread's row: entry i of tile `tile`; the next tile's ray and normals
  // are gathered while this tile runs, its hit record one tile earlier
  auto row_of = [&](int tl) { return tl * kRows + c.t; };
  auto valid = [&](int tl) { return tl < ntiles && row_of(tl) < n; };
  InferRow cur{}, nxt{};
  cur.h = valid(tile) ? I.hits[row_of(tile)] : miss_hit();
  infer_gather(I, row_of(tile), cur);
  nxt.h = valid(tile + step) ? I.hits[row_of(tile + step)] : miss_hit();
  for (; tile < ntiles; tile += step) {
    int const i = row_of(tile);
    float f[6];
    infer_features(I, cur, f);
    if (valid(tile + step)) infer_gather(I, row_of(tile + step), nxt);
    float4 const h2 = valid(tile + 2 * step) ? I.hits[row_of(tile + 2 * step)] : miss_hit();
    float o[kW];
    if (!forward_infer(S.wt, G, c, phase, f, o)) {
      if (c.t == 0) atomicExch(G.err, 1);
      aborted = true;
      break;
    }
    if (i < n) {
      // mixture values (weight, kappa, mean xyz per lobe) packed as fp16
      // pairs in registers; the renderer renormalises what it reads, so the
      // fast intrinsics here only shape the proposal
      float mx = o[0];
#pragma unroll
      for (int j = 1; j < 8; ++j) mx = fmaxf(mx, o[j]);
      float e[8], se = 0.0f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        e[j] = __expf(o[j] - mx);
        se += e[j];
      }
      float const inv_se = 1.0f / se;
      float hv[40];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float const x = o[16 + 3 * j], y = o[17 + 3 * j], z = o[18 + 3 * j];
        float const r = rsqrtf(x * x + y * y + z * z + 1e-12f);
        hv[5 * j] = e[j] * inv_se;
        hv[5 * j + 1] = __expf(fminf(fmaxf(o[8 + j], -5.0f), 8.0f));
        hv[5 * j + 2] = x * r;
        hv[5 * j + 3] = y * r;
        hv[5 * j + 4] = z * r;
      }
      uint32_t wv[20];
#pragma unroll
      for (int t = 0; t < 20; ++t) {
        __half2 const h2 = __floats2half2_rn(hv[2 * t], hv[2 * t + 1]);
        wv[t] = *reinterpret_cast<const uint32_t *>(&h2);
      }
      uint4 *dst = reinterpret_cast<uint4 *>(I.mix + 40 * static_cast<int64_t>(i));
#pragma unroll
      for (int t = 0; t < 5; ++t) dst[t] = make_uint4(wv[4 * t], wv[4 * t + 1], wv[4 * t + 2], wv[4 * t + 3]);
    }
    cur = nxt;
    nxt = InferRow{};
    nxt.h = h2;
  }
  teardown(S.tmem, 256, aborted, c.mbar, phase);
}

// Training records of a guided wave -> (position, normal, direction, weight)
// rows: weight = Y of the incident radiance estimate along the sampled
// direction, (L_path - L_before) / throughput, times the cosine, over the
// sampling density.  Rows with no weight are dropped.
__global__ void k_guide_records(const float *__restrict__ rec, int tb, int64_t npaths,
                                const float4 *__restrict__ radiance, float *__restrict__ out, int *count,
                                int64_t cap) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < npaths * tb;
       idx += stride) {
    const float *r = rec + idx * 16;
    float const q = r[9];
    if (!(q > 0.0f) || isnan(r[14]) || !(r[11] > 0.0f)) continue;
    float4 const L = radiance[idx / tb];
    float const li = (L.y - r[14]) / r[11];
    float const cs = r[3] * r[6] + r[4] * r[7] + r[5] * r[8];
    float const w = li * cs / q;
    if (!(w > 0.0f) || !isfinite(w)) continue;
    int const j = atomicAdd(count, 1);
    if (j >= cap) continue;
    float *o = out + 10 * static_cast<int64_t>(j);
    for (int t = 0; t < 9; ++t) o[t] = r[t];
    o[9] = w;
  }
}

// fp32 master parameters -> the weight image: blocked bf16 W^T per layer, the
// ones tile (128 x 16, columns 0..2 = 1) and per layer the bias tile (64 x 16,
// columns 0..2 = the bias's hi, mid and lo bf16 parts, whose sum is the fp32
// bias to within fp32 rounding).  One thread per image element.
constexpr int kPackWeights = kParams - kLayers * kW;
constexpr int kPackOnes = kRows * kBiasK;
constexpr int kPackBias = kLayers * kW * kBiasK;
constexpr int kPackThreads = kPackWeights + kPackOnes + kPackBias;

__global__ void k_guide_pack(const float *__restrict__ params, uint8_t *__restrict__ wblk) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kPackWeights) {
    int l = 0, rem = i;
    while (l < kLayers && rem >= layer_in(l) * kW) {
      rem -= layer_in(l) * kW;
      ++l;
    }
    int const K = layer_in(l);
    int const k = rem / kW, nn = rem % kW;  // W_l[k][nn]
    __nv_bfloat16 const b = __float2bfloat16_rn(params[param_w(l) + k * kW + nn]);
    *reinterpret_cast<__nv_bfloat16 *>(wblk + wblk_off(l) + tc::blocked_offset(nn, k, K)) = b;
  } else if (i < kPackWeights + kPackOnes) {
    int const j = i - kPackWeights;
    int const r = j / kBiasK, c = j % kBiasK;
    *reinterpret_cast<__nv_bfloat16 *>(wblk + kOnesOff + tc::blocked_offset(r, c, kBiasK)) =
        __float2bfloat16_rn(c < 3 ? 1.0f : 0.0f);
  } else if (i < kPackThreads) {
    int const j = i - kPackWeights - kPackOnes;
    int const l = j / (kW * kBiasK), n = (j / kBiasK) % kW, c = j % kBiasK;
    float const b = params[param_b(l) + n];
    __nv_bfloat16 const hi = __float2bfloat16_rn(b);
    float const r1 = b - __bfloat162float(hi);
    __nv_bfloat16 const mid = __float2bfloat16_rn(r1);
    __nv_bfloat16 const lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
    __nv_bfloat16 const v = c == 0 ? hi : c == 1 ? mid : c == 2 ? lo : __float2bfloat16_rn(0.0f);
    *reinterpret_cast<__nv_bfloat16 *>(wblk + kBiasOff + l * (kW * kBiasK * 2) + tc::blocked_offset(n, c, kBiasK)) = v;
  }
}

// One Adam step (bias-corrected, fp32 masters) fused with the re-pack of the
// changed values into the weight image: a weight's bf16 copy in the blocked
// W^T layout, a bias's hi / mid / lo parts in its bias tile (the ones tile and
// the bias tiles' zero columns never change; k_guide_pack writes them).  The
// step number comes from the training state: t = ts->step + step_rel + 1.
// gate: skip the step when the training pass produced no rows.
__global__ void k_guide_adam_pack(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m,
                                  float *__restrict__ v, uint8_t *__restrict__ wblk, float lr, float eps,
                                  const TrainState *__restrict__ ts, int step_rel, long long cap, int gate) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  if (gate && min(static_cast<long long>(ts->count), cap) <= 0) return;
  long long const t = ts->step + step_rel + 1;
  float const b1 = 0.9f, b2 = 0.99f;
  float const c1 = static_cast<float>(1.0 - pow(0.9, static_cast<double>(t)));
  float const c2 = static_cast<float>(1.0 - pow(0.99, static_cast<double>(t)));
  float const gi = g[i];
  float const mi = b1 * m[i] + (1.0f - b1) * gi;
  float const vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float const pn = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pn;
  g[i] = 0.0f;
  // position of parameter i in the image
  int l = 0, rem = i;
  while (l < kLayers && rem >= layer_in(l) * kW + kW) {
    rem -= layer_in(l) * kW + kW;
    ++l;
  }
  int const K = layer_in(l);
  if (rem < K * kW) {
    int const k = rem / kW, nn = rem % kW;  // W_l[k][nn]
    *reinterpret_cast<__nv_bfloat16 *>(wblk + wblk_off(l) + tc::blocked_offset(nn, k, K)) = __float2bfloat16_rn(pn);
  } else {
    int const nn = rem - K * kW;  // b_l[nn]
    __nv_bfloat16 const hi = __float2bfloat16_rn(pn);
    float const r1 = pn - __bfloat162float(hi);
    __nv_bfloat16 const mid = __float2bfloat16_rn(r1);
    __nv_bfloat16 const lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
    uint8_t *const base = wblk + kBiasOff + l * (kW * kBiasK * 2);
    *reinterpret_cast<__nv_bfloat16 *>(base + tc::blocked_offset(nn, 0, kBiasK)) = hi;
    *reinterpret_cast<__nv_bfloat16 *>(base + tc::blocked_offset(nn, 1, kBiasK)) = mid;
    *reinterpret_cast<__nv_bfloat16 *>(base + tc::blocked_offset(nn, 2, kBiasK)) = lo;
  }
}

// Bookkeeping after Adam steps.  pass: a training pass over min(count, cap)
// rows took `steps` steps of min(batch, rows) rows (nothing happened if there
// were no rows); else `steps` explicit steps.
__global__ void k_guide_advance(TrainState *ts, int steps, int batch, long long cap, int pass) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!pass) {
    ts->step += steps;
    return;
  }
  long long const rows = min(static_cast<long long>(ts->count), cap);
  if (rows <= 0) return;
  long long const bs = min(static_cast<long long>(batch), rows);
  ts->offset += static_cast<long long>(steps) * bs;
  ts->step += steps;
  ts->trained += static_cast<unsigned long long>(rows);
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
  TrainState *d_ts = nullptr;  // Adam step, batch offset, row counts (device)
  float lo[3] = {0, 0, 0}, inv_ext[3] = {1, 1, 1};
  // guided-render buffers
  __half *d_mix = nullptr;
  int64_t mix_cap = 0;
  float *d_rec = nullptr, *d_train = nullptr;
  int64_t rec_cap = 0;  // paths
  // One CUDA graph per training-pass shape (records kernel, steps_per_pass x
  // (gradient, Adam + pack), bookkeeping), captured on a private stream the
  // first time a wave of that size trains and replayed on the caller's stream.
  struct Pass {
    int64_t npaths;
    const float4 *radiance;
    cudaGraphExec_t exec;
  };
  std::vector<Pass> passes;
  cudaStream_t cap_st = nullptr;
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
  k_guide_pack<<<(kPackThreads + 255) / 256, 256, 0, st>>>(g.d_params, g.d_wblk);
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
                                      static_cast<int>(sizeof(InferSmem))));
    attr = true;
  }
  if (n <= 0) return XYZGPU_OK;
  int const grid = std::max(1, std::min((n + kGroups * kRows - 1) / (kGroups * kRows), sm_count(g.device)));
  k_guide_forward<<<grid, kInferThreads, sizeof(InferSmem), st>>>(guide_dev(g), feat, n, out);
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
  GradArgs A{rec, n, scale, grad, nullptr, 0, 0, 0};
  k_guide_gradient<<<grid_for(g.device, n), kGuideThreads, sizeof(GuideSmem), st>>>(guide_dev(g), A);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

void drop_passes(GuideImpl &g) {
  for (auto &p : g.passes) cudaGraphExecDestroy(p.exec);
  g.passes.clear();
}

int guide_wave_prepare(GuideImpl &g, int64_t cap, bool train, cudaStream_t st, GuideWave *out) {
  if (g.mix_cap < cap) {
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(g.d_mix);
    g.d_mix = nullptr;
    g.mix_cap = 0;
    cudaError_t const e = cudaMalloc(reinterpret_cast<void **>(&g.d_mix), static_cast<size_t>(cap) * 40 * sizeof(__half));
    if (e != cudaSuccess) return set_error(XYZGPU_E_NOMEM, "render_guided: mixture buffer: %s", cudaGetErrorString(e));
    g.mix_cap = cap;
  }
  int const tb = g.cfg.train_bounces;
  if (train && tb > 0 && g.rec_cap < cap) {
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    drop_passes(g);
    cudaFree(g.d_rec);
    cudaFree(g.d_train);
    g.d_rec = g.d_train = nullptr;
    g.rec_cap = 0;
    size_t const n = static_cast<size_t>(cap) * tb;
    if (cudaMalloc(reinterpret_cast<void **>(&g.d_rec), n * 16 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&g.d_train), n * 10 * sizeof(float)) != cudaSuccess)
      return set_error(XYZGPU_E_NOMEM, "render_guided: training record buffers of %zu records", n);
    g.rec_cap = cap;
  }
  out->mix = g.d_mix;
  out->records = train && tb > 0 ? g.d_rec : nullptr;
  out->train_bounces = train ? tb : 0;
  out->alpha = g.cfg.alpha;
  out->guide_bounces = g.cfg.guide_bounces;
  return XYZGPU_OK;
}

int guide_infer_launch(GuideImpl &g, const float4 *qo, const float4 *qd, const float4 *hits,
                       const int32_t *count, const DevScene &S, void *mix, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    XYZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(sizeof(InferSmem))));
    attr = true;
  }
  InferArgs I{qo, qd, hits, count, S.tri_ng, S.tri_sn, static_cast<__half *>(mix)};
  k_guide_infer<<<sm_count(g.device), kInferThreads, sizeof(InferSmem), st>>>(guide_dev(g), I);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int adam_pack_launch(GuideImpl &g, const GuideDev &, int step_rel, long long cap, int gate, cudaStream_t st) {
  k_guide_adam_pack<<<(kParams + 255) / 256, 256, 0, st>>>(g.d_params, g.d_grad, g.d_m, g.d_v, g.d_wblk,
                                                          g.cfg.learning_rate, 1e-8f, g.d_ts, step_rel, cap, gate);
  return cudaGetLastError() == cudaSuccess ? XYZGPU_OK : set_error(XYZGPU_E_CUDA, "guide: Adam launch failed");
}

// Enqueues a training pass's launches on `st` (which is being captured).
int enqueue_pass(GuideImpl &g, const float4 *radiance, int64_t npaths, cudaStream_t st) {
  int const tb = g.cfg.train_bounces;
  long long const cap = npaths * tb;
  GuideDev const G = guide_dev(g);
  XYZ_CUDA_TRY(cudaMemsetAsync(&g.d_ts->count, 0, sizeof(int), st));
  int const blocks = std::max(1, std::min<int>(static_cast<int>((cap + 255) / 256), sm_count(g.device) * 8));
  k_guide_records<<<blocks, 256, 0, st>>>(g.d_rec, tb, npaths, radiance, g.d_train, &g.d_ts->count, cap);
  XYZ_CUDA_TRY(cudaGetLastError());
  // every CTA of the gradient grid takes tiles of the batch; the batch size
  // is known only on the device, so the grid is one CTA per SM
  int const grid = std::max(1, std::min(sm_count(g.device), (g.cfg.batch_size + kRows - 1) / kRows));
  for (int s = 0; s < g.cfg.steps_per_pass; ++s) {
    GradArgs A{g.d_train, 0, 0.0f, g.d_grad, g.d_ts, cap, s, g.cfg.batch_size};
    k_guide_gradient<<<grid, kGuideThreads, sizeof(GuideSmem), st>>>(G, A);
    XYZ_CUDA_TRY(cudaGetLastError());
    int const rc = adam_pack_launch(g, G, s, cap, 1, st);
    if (rc) return rc;
  }
  k_guide_advance<<<1, 32, 0, st>>>(g.d_ts, g.cfg.steps_per_pass, g.cfg.batch_size, cap, 1);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

// After a training wave: records -> training rows, then steps_per_pass Adam
// steps on batches of batch_size rows (cycling through the rows), all on the
// device: one graph launch, no host synchronisation.
int guide_train_on_wave(GuideImpl &g, const float4 *radiance, int64_t npaths, cudaStream_t st) {
  int const tb = g.cfg.train_bounces;
  if (tb <= 0 || g.cfg.steps_per_pass <= 0 || !g.d_rec) return XYZGPU_OK;
  cudaGraphExec_t exec = nullptr;
  for (auto &p : g.passes)
    if (p.npaths == npaths && p.radiance == radiance) exec = p.exec;
  if (!exec) {
    static bool attr = false;
    if (!attr) {
      XYZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_gradient, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(sizeof(GuideSmem))));
      attr = true;
    }
    if (!g.cap_st) XYZ_CUDA_TRY(cudaStreamCreateWithFlags(&g.cap_st, cudaStreamNonBlocking));
    if (g.passes.size() >= 4) drop_passes(g);
    XYZ_CUDA_TRY(cudaStreamBeginCapture(g.cap_st, cudaStreamCaptureModeThreadLocal));
    int const rc = enqueue_pass(g, radiance, npaths, g.cap_st);
    cudaGraph_t graph = nullptr;
    cudaError_t const e = cudaStreamEndCapture(g.cap_st, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return set_error(XYZGPU_E_CUDA, "render_guided: capturing the training pass: %s",
                                           cudaGetErrorString(e));
    cudaError_t const ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return set_error(XYZGPU_E_CUDA, "render_guided: instantiating the training pass: %s",
                                            cudaGetErrorString(ei));
    g.passes.push_back(GuideImpl::Pass{npaths, radiance, exec});
  }
  XYZ_CUDA_TRY(cudaGraphLaunch(exec, st));
  return XYZGPU_OK;
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
  c->guide_bounces = 4;
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
  cudaFree(g.d_mix);
  cudaFree(g.d_rec);
  cudaFree(g.d_train);
  cudaFree(g.d_ts);
  drop_passes(g);
  if (g.cap_st) cudaStreamDestroy(g.cap_st);
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
      c.steps_per_pass < 0 || c.train_bounces < 0 || c.train_bounces > 8 || c.guide_bounces < 0)
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
      cudaMalloc(reinterpret_cast<void **>(&g.d_wblk), kWImageBytes) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_err), sizeof(int)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void **>(&g.d_ts), sizeof(TrainState)) != cudaSuccess)
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
      cudaMemset(g.d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaMemset(g.d_ts, 0, sizeof(TrainState)) != cudaSuccess)
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
  XYZ_CUDA_TRY(cudaMemset(&g.d_ts->step, 0, sizeof(long long)));
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

int xyzgpu_render_guided(xyzgpu_guide h, const xyzgpu_camera *cam, const xyzgpu_render_params *rp, int train,
                         float *film, void *stream) {
  clear_error();
  if (!h || !cam || !rp || !film) return set_error(XYZGPU_E_INVALID, "render_guided: null argument");
  if (rp->spectral != XYZGPU_SPECTRAL_OFF || (rp->profile != XYZGPU_PROFILE_OFF && rp->profile != XYZGPU_PROFILE_TIMING))
    return set_error(XYZGPU_E_INVALID, "render_guided: the XYZ film mode only, profile off or timing");
  if (rp->width <= 0 || rp->height <= 0 || rp->spp < 0 || rp->spp_offset < 0 || rp->max_depth < 1 ||
      rp->max_depth > 1000 || rp->rr_start_depth < 1 || !(rp->rr_threshold >= 0.0f) || rp->wave_paths < 0 ||
      (rp->film_location != XYZGPU_FILM_DEVICE && rp->film_location != XYZGPU_FILM_HOST) ||
      !((rp->row_begin == 0 && rp->row_end == 0) ||
        (rp->row_begin >= 0 && rp->row_begin < rp->row_end && rp->row_end <= rp->height)) ||
      rp->row_step < 0)
    return set_error(XYZGPU_E_INVALID, "render_guided: parameters out of range");
  if (static_cast<int64_t>(rp->width) * rp->height >= (1ll << 31) ||
      static_cast<int64_t>(rp->spp_offset) + rp->spp >= (1ll << 32))
    return set_error(XYZGPU_E_LIMIT, "render_guided: image or sample index too large");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(cam->eye[k]) || !std::isfinite(cam->at[k]))
      return set_error(XYZGPU_E_INVALID, "render_guided: camera position is not finite");
  if (!(cam->film_size > 0) || !(cam->focal_length > 0) || !(cam->f_number > 0))
    return set_error(XYZGPU_E_INVALID, "render_guided: camera film size, focal length and F-number must be > 0");
  GuideImpl &g = h->g;
  if (g.scene->n_specular)
    return set_error(XYZGPU_E_INVALID, "render_guided: scenes with mirror or metal materials are not guided");
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  XYZ_CUDA_TRY(cudaMemsetAsync(g.d_err, 0, sizeof(int), st));
  GuideHooks hooks{&g, train != 0};
  int const rc = render_launch(*g.scene, *cam, *rp, film, st, nullptr, &hooks);
  if (rc) return rc;
  return check_err(g, st, "render_guided");
}

int xyzgpu_guide_stats_get(xyzgpu_guide h, xyzgpu_guide_stats *out) {
  clear_error();
  if (!h || !out) return set_error(XYZGPU_E_INVALID, "guide_stats_get: null argument");
  XYZ_CUDA_TRY(cudaSetDevice(h->g.device));
  XYZ_CUDA_TRY(cudaDeviceSynchronize());
  TrainState ts;
  XYZ_CUDA_TRY(cudaMemcpy(&ts, h->g.d_ts, sizeof(ts), cudaMemcpyDeviceToHost));
  out->adam_steps = static_cast<uint64_t>(ts.step);
  out->trained_records = ts.trained;
  return XYZGPU_OK;
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
  rc = adam_pack_launch(g, guide_dev(g), 0, 0, 0, st);
  if (rc) return rc;
  k_guide_advance<<<1, 32, 0, st>>>(g.d_ts, 1, 0, 0, 0);
  XYZ_CUDA_TRY(cudaGetLastError());
  return check_err(g, st, "guide_train_step");
}

int xyzgpu_guide_reserve(xyzgpu_guide h, int64_t wave_paths, int train, void *stream) {
  clear_error();
  if (!h || wave_paths <= 0) return set_error(XYZGPU_E_INVALID, "guide_reserve: bad argument");
  if (wave_paths > (int64_t{1} << 23))
    return set_error(XYZGPU_E_LIMIT, "guide_reserve: at most 2^23 paths per guided wave");
  GuideImpl &g = h->g;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  XYZ_CUDA_TRY(cudaSetDevice(g.device));
  GuideWave gw;
  int const rc = guide_wave_prepare(g, wave_paths, train != 0, st, &gw);
  if (rc) return rc;
  XYZ_CUDA_TRY(cudaStreamSynchronize(st));
  return XYZGPU_OK;
}

}  // extern "C"
