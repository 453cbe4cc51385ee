// Film output on the device and the file formats around it:
//  * the Radiance RGBE pixel encoding of ImageFilm::SaveAsHdr
//    (xyz/core/imagefilm_hdr.cpp:14-31, 124-183) as a kernel, and the file
//    (header and run-length scanlines, :46-114) written on the host;
//  * the float2bmp tone operators (float2bmp/main.cpp:69-118, 209-214) as a
//    kernel producing 24-bit BMP pixel rows, and the BMP file;
//  * a resumable render checkpoint: film sums, the number of samples done
//    and the render parameters, so a render continues where it stopped (the
//    reference's periodic .pfm dump, xyz/integrator/integrator.cpp:140-160,
//    keeps the image but not a way to continue it).
// All three read the film as xyzgpu_render leaves it: W * H XYZ sums, row 0
// at the bottom.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "scene.h"

namespace xyzgpu {
namespace {

constexpr int kFilmThreads = 256;

int film_grid(int64_t n) {
  int dev = 0;
  cudaGetDevice(&dev);
  int64_t const want = (n + kFilmThreads - 1) / kFilmThreads;
  int64_t const cap = static_cast<int64_t>(sm_count(dev)) * 8;
  return static_cast<int>(std::max<int64_t>(1, std::min(want, cap)));
}

// static_cast<unsigned char>(float) as the reference's build performs it: the
// value truncated towards zero to a 32-bit integer, whose low byte is kept
// (negative colour components of saturated XYZ wrap around rather than
// saturate).
__device__ __forceinline__ uint8_t byte_of(float v) { return static_cast<uint8_t>(static_cast<uint32_t>(__float2int_rz(v))); }

// hdr_encode (imagefilm_hdr.cpp:14-31): mantissa scale frexp(d) * 255.9999 / d
// in double, rounded to float, times each component.
__device__ __forceinline__ uchar4 rgbe_of(float r, float g, float b) {
  float const d = fmaxf(fmaxf(r, g), b);
  if (static_cast<double>(d) <= 1e-32) return make_uchar4(0, 0, 0, 0);
  int e = 0;
  float const m = frexpf(d, &e);
  float const f = static_cast<float>(static_cast<double>(m) * 255.9999 / static_cast<double>(d));
  return make_uchar4(byte_of(r * f), byte_of(g * f), byte_of(b * f), static_cast<uint8_t>(e + 128));
}

// One thread per pixel; output in file order.  RGBE: scanlines from the top
// image row down ("-Y H +X W"), the film's XYZ / spp converted to CCIR 601-1
// RGB (CCIR601_1_XYZ2RGB, libhi/hi/image/color_space.hpp:69-79) and a
// non-finite pixel written as 0.  XYZE (the reference's CONFIG_HDR_STRICT
// build): XYZ / spp, scanlines from the bottom row up ("+Y H +X W").
__global__ void k_film_rgbe(const float *__restrict__ film, int W, int H, float scale, int xyze,
                            uchar4 *__restrict__ out) {
  int64_t const n = static_cast<int64_t>(W) * H;
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t const row = q / W, x = q - row * W;
    int64_t const p = (xyze ? row : (H - 1 - row)) * W + x;
    float const X = film[3 * p] * scale, Y = film[3 * p + 1] * scale, Z = film[3 * p + 2] * scale;
    if (xyze) {
      out[q] = rgbe_of(X, Y, Z);
      continue;
    }
    float r = 1.9104f * X - 0.5338f * Y - 0.2891f * Z;
    float g = -0.9844f * X + 1.9985f * Y - 0.0279f * Z;
    float b = 0.0585f * X - 0.1187f * Y + 0.9017f * Z;
    if (!isfinite(r) || !isfinite(g) || !isfinite(b)) r = g = b = 0.0f;
    out[q] = rgbe_of(r, g, b);
  }
}

// float2bmp's luminance for the white point of the Reinhard operator: the
// maximum over pixels of 0.6069 c0 + 0.1735 c1 + 0.2003 c2 of the values
// tone-mapped (float2bmp/main.cpp:186-196; the maximum starts at 0, so the
// non-negative float bits order as integers).
__global__ void k_film_max_luminance(const float *__restrict__ film, int64_t n, float scale, int rgb,
                                     unsigned int *out) {
  float best = 0.0f;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float c[3] = {film[3 * p] * scale, film[3 * p + 1] * scale, film[3 * p + 2] * scale};
    if (rgb) {
      float const X = c[0], Y = c[1], Z = c[2];
      c[0] = 1.9104f * X - 0.5338f * Y - 0.2891f * Z;
      c[1] = -0.9844f * X + 1.9985f * Y - 0.0279f * Z;
      c[2] = 0.0585f * X - 0.1187f * Y + 0.9017f * Z;
    }
    float const l = 0.6069f * c[0] + 0.1735f * c[1] + 0.2003f * c[2];
    if (best < l) best = l;
  }
  for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_down_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best > 0.0f) atomicMax(out, __float_as_uint(best));
}

struct ToneArgs {
  float scale, exposure, white, gamma;
  int op, rgb;
  const unsigned int *white_bits;  // device maximum luminance (white <= 0), else null
};

// tonemap() of float2bmp/main.cpp:80-118: operator, gamma src / dst, then the
// 8-bit quantisation of clamp() (:69-77).
__device__ __forceinline__ uint8_t tone_one(float light, const ToneArgs &T, float white) {
  if (light <= 0.0f) return 0;
  float v;
  switch (T.op) {
    case XYZGPU_TONEMAP_LINEAR: v = T.exposure * light; break;
    case XYZGPU_TONEMAP_REINHARD: v = T.exposure * light / (1.0f + light); break;
    case XYZGPU_TONEMAP_REINHARD_WHITE: v = T.exposure * light * (1.0f + light / (white * white)) / (1.0f + light); break;
    default: v = 1.0f - expf(-T.exposure * light); break;
  }
  v = powf(v, T.gamma);
  if (v <= 0.0f) return 0;
  if (v >= 1.0f) return 255;
  return static_cast<uint8_t>(v * 256.0f);
}

// One thread per pixel; BMP order (rows from the bottom, as the film) and
// byte order (blue, green, red = channel 2, 1, 0), rows padded to 4 bytes.
__global__ void k_film_tonemap(const float *__restrict__ film, int W, int H, ToneArgs T, uint8_t *__restrict__ out) {
  float const white = T.white_bits ? __uint_as_float(*T.white_bits) : T.white;
  int64_t const stride_b = (3 * static_cast<int64_t>(W) + 3) & ~int64_t{3};
  int64_t const n = static_cast<int64_t>(W) * H;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float c[3] = {film[3 * p] * T.scale, film[3 * p + 1] * T.scale, film[3 * p + 2] * T.scale};
    if (T.rgb) {
      float const X = c[0], Y = c[1], Z = c[2];
      c[0] = 1.9104f * X - 0.5338f * Y - 0.2891f * Z;
      c[1] = -0.9844f * X + 1.9985f * Y - 0.0279f * Z;
      c[2] = 0.0585f * X - 0.1187f * Y + 0.9017f * Z;
    }
    int64_t const y = p / W, x = p - y * W;
    uint8_t *o = out + y * stride_b + 3 * x;
    o[2] = tone_one(c[0], T, white);
    o[1] = tone_one(c[1], T, white);
    o[0] = tone_one(c[2], T, white);
    // the row's padding bytes are zero (the caller's buffer may hold anything)
    if (x == W - 1)
      for (int64_t b = 3 * static_cast<int64_t>(W); b < stride_b; ++b) out[y * stride_b + b] = 0;
  }
}

// ---- Radiance run-length scanline (the format of imagefilm_hdr.cpp:46-114):
// lines of 8..32767 pixels start with 2, 2, width (16 bits, big-endian) and
// hold each of the four byte planes as packets: a run (128 + n, value) of
// n = 4..127 equal bytes or a literal (n, then n bytes) of n = 1..128 bytes;
// shorter runs stay inside literals.  Other widths are written flat.
void write_rle_line(const uint8_t *px, int W, std::vector<uint8_t> &o) {
  if (W < 8 || W > 0x7fff) {
    o.insert(o.end(), px, px + 4 * static_cast<size_t>(W));
    return;
  }
  o.push_back(2);
  o.push_back(2);
  o.push_back(static_cast<uint8_t>((W >> 8) & 0xff));
  o.push_back(static_cast<uint8_t>(W & 0xff));
  for (int c = 0; c < 4; ++c) {
    auto at = [&](int i) { return px[4 * i + c]; };
    int lit = 0;  // start of the pending literal bytes
    int i = 0;
    auto flush = [&](int end) {
      while (lit < end) {
        int const n = std::min(128, end - lit);
        o.push_back(static_cast<uint8_t>(n));
        for (int k = 0; k < n; ++k) o.push_back(at(lit + k));
        lit += n;
      }
    };
    while (i < W) {
      int run = 1;
      while (run < 127 && i + run < W && at(i + run) == at(i)) ++run;
      if (run >= 4) {
        flush(i);
        o.push_back(static_cast<uint8_t>(128 + run));
        o.push_back(at(i));
        i += run;
        lit = i;
      } else {
        i += run;
      }
    }
    flush(W);
  }
}

uint64_t fnv1a(const void *p, size_t n, uint64_t h = 1469598103934665603ull) {
  const uint8_t *b = static_cast<const uint8_t *>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

constexpr char kCkptMagic[8] = {'X', 'Y', 'Z', 'G', 'P', 'U', 'C', 'K'};
constexpr uint32_t kCkptVersion = 1;

}  // namespace
}  // namespace xyzgpu

using namespace xyzgpu;

extern "C" {

int xyzgpu_film_encode_rgbe(const float *film, int width, int height, float scale, int xyze, uint8_t *out,
                            void *stream) {
  clear_error();
  if (!film || !out || width <= 0 || height <= 0 || !std::isfinite(scale))
    return set_error(XYZGPU_E_INVALID, "film_encode_rgbe: bad argument");
  int64_t const n = static_cast<int64_t>(width) * height;
  k_film_rgbe<<<film_grid(n), kFilmThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      film, width, height, scale, xyze != 0, reinterpret_cast<uchar4 *>(out));
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int xyzgpu_hdr_write(const char *path, const uint8_t *rgbe, int width, int height, int xyze) {
  clear_error();
  if (!path || !rgbe || width <= 0 || height <= 0) return set_error(XYZGPU_E_INVALID, "hdr_write: bad argument");
  std::vector<uint8_t> o;
  char head[256];
  int const hn = std::snprintf(head, sizeof(head),
                               "#?RADIANCE\n# Made with xyzgpu\nFORMAT=32-bit_rle_%s\nEXPOSURE=1.0000000000000\n\n"
                               "%cY %d +X %d\n",
                               xyze ? "xyze" : "rgbe", xyze ? '+' : '-', height, width);
  o.insert(o.end(), head, head + hn);
  for (int r = 0; r < height; ++r) write_rle_line(rgbe + 4 * static_cast<size_t>(r) * width, width, o);
  FILE *f = std::fopen(path, "wb");
  if (!f) return set_error(XYZGPU_E_INVALID, "hdr_write: cannot open %s", path);
  size_t const w = std::fwrite(o.data(), 1, o.size(), f);
  if (std::fclose(f) != 0 || w != o.size()) return set_error(XYZGPU_E_INVALID, "hdr_write: writing %s failed", path);
  return XYZGPU_OK;
}

void xyzgpu_tonemap_params_default(xyzgpu_tonemap_params *tp) {
  if (!tp) return;
  tp->scale = 1.0f;
  tp->op = XYZGPU_TONEMAP_FILM;
  tp->exposure = 1.0f;
  tp->white = 0.0f;
  tp->dst_gamma = 2.2f;
  tp->src_gamma = 1.0f;
  tp->rgb = 0;
}

int xyzgpu_film_tonemap(const float *film, int width, int height, const xyzgpu_tonemap_params *tp, uint8_t *out,
                        unsigned int *scratch_white, void *stream) {
  clear_error();
  if (!film || !out || !tp || width <= 0 || height <= 0 || !std::isfinite(tp->scale) ||
      !std::isfinite(tp->exposure) || !(tp->dst_gamma > 0.0f) || !(tp->src_gamma > 0.0f) || tp->op < 0 ||
      tp->op > XYZGPU_TONEMAP_REINHARD_WHITE)
    return set_error(XYZGPU_E_INVALID, "film_tonemap: bad argument");
  bool const need_white = tp->op == XYZGPU_TONEMAP_REINHARD_WHITE && !(tp->white > 0.0f);
  if (need_white && !scratch_white)
    return set_error(XYZGPU_E_INVALID, "film_tonemap: the image's white point needs a device word (scratch_white)");
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  int64_t const n = static_cast<int64_t>(width) * height;
  ToneArgs T{tp->scale, tp->exposure, tp->white, tp->src_gamma / tp->dst_gamma, tp->op, tp->rgb != 0, nullptr};
  if (need_white) {
    XYZ_CUDA_TRY(cudaMemsetAsync(scratch_white, 0, sizeof(unsigned int), st));
    k_film_max_luminance<<<film_grid(n), kFilmThreads, 0, st>>>(film, n, tp->scale, tp->rgb != 0, scratch_white);
    T.white_bits = scratch_white;
  }
  k_film_tonemap<<<film_grid(n), kFilmThreads, 0, st>>>(film, width, height, T, out);
  XYZ_CUDA_TRY(cudaGetLastError());
  return XYZGPU_OK;
}

int xyzgpu_bmp_write(const char *path, const uint8_t *bgr, int width, int height) {
  clear_error();
  if (!path || !bgr || width <= 0 || height <= 0) return set_error(XYZGPU_E_INVALID, "bmp_write: bad argument");
  uint32_t const stride = (3u * static_cast<uint32_t>(width) + 3u) & ~3u;
  uint32_t const data = stride * static_cast<uint32_t>(height);
  uint8_t h[54] = {0};
  auto put32 = [&](int at, uint32_t v) {
    for (int k = 0; k < 4; ++k) h[at + k] = static_cast<uint8_t>(v >> (8 * k));
  };
  h[0] = 'B';
  h[1] = 'M';
  put32(2, 54 + data);                        // file size
  put32(10, 54);                              // pixel data offset
  put32(14, 40);                              // BITMAPINFOHEADER size
  put32(18, static_cast<uint32_t>(width));
  put32(22, static_cast<uint32_t>(height));   // positive: rows from the bottom
  h[26] = 1;                                  // planes
  h[28] = 24;                                 // bits per pixel, BI_RGB
  FILE *f = std::fopen(path, "wb");
  if (!f) return set_error(XYZGPU_E_INVALID, "bmp_write: cannot open %s", path);
  bool ok = std::fwrite(h, 1, 54, f) == 54 && std::fwrite(bgr, 1, data, f) == data;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? XYZGPU_OK : set_error(XYZGPU_E_INVALID, "bmp_write: writing %s failed", path);
}

// Host-film conveniences: upload, device encode / tone map, write the file.
int xyzgpu_film_save_hdr(const char *path, const float *film, int width, int height, float spp, int xyze) {
  clear_error();
  if (!path || !film || width <= 0 || height <= 0 || !(spp > 0.0f))
    return set_error(XYZGPU_E_INVALID, "film_save_hdr: bad argument");
  size_t const n = static_cast<size_t>(width) * height;
  float *d_film = nullptr;
  uint8_t *d_px = nullptr;
  struct Free {
    float *&a;
    uint8_t *&b;
    ~Free() {
      cudaFree(a);
      cudaFree(b);
    }
  } guard{d_film, d_px};
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&d_film), 3 * n * sizeof(float)));
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&d_px), 4 * n));
  XYZ_CUDA_TRY(cudaMemcpy(d_film, film, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  int rc = xyzgpu_film_encode_rgbe(d_film, width, height, 1.0f / spp, xyze, d_px, nullptr);
  if (rc) return rc;
  std::vector<uint8_t> px(4 * n);
  XYZ_CUDA_TRY(cudaMemcpy(px.data(), d_px, 4 * n, cudaMemcpyDeviceToHost));
  return xyzgpu_hdr_write(path, px.data(), width, height, xyze);
}

int xyzgpu_film_save_bmp(const char *path, const float *film, int width, int height,
                         const xyzgpu_tonemap_params *tp) {
  clear_error();
  if (!path || !film || !tp || width <= 0 || height <= 0)
    return set_error(XYZGPU_E_INVALID, "film_save_bmp: bad argument");
  size_t const n = static_cast<size_t>(width) * height;
  size_t const bytes = ((3 * static_cast<size_t>(width) + 3) & ~size_t{3}) * height;
  float *d_film = nullptr;
  uint8_t *d_px = nullptr;
  unsigned int *d_white = nullptr;
  struct Free {
    float *&a;
    uint8_t *&b;
    unsigned int *&c;
    ~Free() {
      cudaFree(a);
      cudaFree(b);
      cudaFree(c);
    }
  } guard{d_film, d_px, d_white};
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&d_film), 3 * n * sizeof(float)));
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&d_px), bytes));
  XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&d_white), sizeof(unsigned int)));
  XYZ_CUDA_TRY(cudaMemcpy(d_film, film, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  int rc = xyzgpu_film_tonemap(d_film, width, height, tp, d_px, d_white, nullptr);
  if (rc) return rc;
  std::vector<uint8_t> px(bytes);
  XYZ_CUDA_TRY(cudaMemcpy(px.data(), d_px, bytes, cudaMemcpyDeviceToHost));
  return xyzgpu_bmp_write(path, px.data(), width, height);
}

int xyzgpu_checkpoint_save(const char *path, const xyzgpu_render_params *rp, int spp_done, const float *film) {
  clear_error();
  if (!path || !rp || !film || rp->width <= 0 || rp->height <= 0 || spp_done < 0)
    return set_error(XYZGPU_E_INVALID, "checkpoint_save: bad argument");
  size_t const n = 3 * static_cast<size_t>(rp->width) * rp->height;
  std::string const tmp = std::string(path) + ".part";
  FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) return set_error(XYZGPU_E_INVALID, "checkpoint_save: cannot open %s", tmp.c_str());
  uint32_t const ver = kCkptVersion, psize = sizeof(xyzgpu_render_params);
  int32_t const done = spp_done;
  uint64_t const sum = fnv1a(film, n * sizeof(float));
  bool ok = std::fwrite(kCkptMagic, 1, 8, f) == 8 && std::fwrite(&ver, 4, 1, f) == 1 &&
            std::fwrite(&psize, 4, 1, f) == 1 && std::fwrite(rp, psize, 1, f) == 1 &&
            std::fwrite(&done, 4, 1, f) == 1 && std::fwrite(&sum, 8, 1, f) == 1 &&
            std::fwrite(film, sizeof(float), n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return set_error(XYZGPU_E_INVALID, "checkpoint_save: writing %s failed", path);
  }
  return XYZGPU_OK;
}

int xyzgpu_checkpoint_load(const char *path, xyzgpu_render_params *rp, int *spp_done, float *film) {
  clear_error();
  if (!path || !rp || !spp_done) return set_error(XYZGPU_E_INVALID, "checkpoint_load: bad argument");
  FILE *f = std::fopen(path, "rb");
  if (!f) return set_error(XYZGPU_E_INVALID, "checkpoint_load: cannot open %s", path);
  char magic[8];
  uint32_t ver = 0, psize = 0;
  int32_t done = 0;
  uint64_t sum = 0;
  xyzgpu_render_params p;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCkptMagic, 8) == 0 &&
            std::fread(&ver, 4, 1, f) == 1 && ver == kCkptVersion && std::fread(&psize, 4, 1, f) == 1 &&
            psize == sizeof(p) && std::fread(&p, psize, 1, f) == 1 && std::fread(&done, 4, 1, f) == 1 &&
            std::fread(&sum, 8, 1, f) == 1 && p.width > 0 && p.height > 0 && done >= 0;
  if (!ok) {
    std::fclose(f);
    return set_error(XYZGPU_E_INVALID, "checkpoint_load: %s is not a checkpoint of this library", path);
  }
  *rp = p;
  *spp_done = done;
  if (film) {
    size_t const n = 3 * static_cast<size_t>(p.width) * p.height;
    ok = std::fread(film, sizeof(float), n, f) == n && fnv1a(film, n * sizeof(float)) == sum;
  }
  std::fclose(f);
  return ok ? XYZGPU_OK : set_error(XYZGPU_E_INVALID, "checkpoint_load: %s is truncated or damaged", path);
}

}  // extern "C"
