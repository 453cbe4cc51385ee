/* Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11), restated for the
 * oracle.  TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's
 * CPU-baseline leg use anything under oracle/.
 *
 * Stream convention shared with the CUDA path (include/xyzgpu.h):
 *   key     = (seed & 0xffffffff, seed >> 32)
 *   counter = (pixel, sample, dim / 4, 0)
 *   u(dim)  = (word[dim % 4] >> 8) * 2^-24          in [0, 1)
 * Dimension d of sample s of pixel p is therefore independent of the order in
 * which paths are traced, which is what lets a CPU and a GPU estimator consume
 * identical numbers path by path. */
#ifndef XYZ_ORACLE_PHILOX_H_
#define XYZ_ORACLE_PHILOX_H_
#include <stdint.h>

static inline void xyzo_philox4x32_10(const uint32_t ctr_in[4], uint32_t k0,
                                      uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

static inline float xyzo_u01(uint32_t w) {
  return (float)(w >> 8) * (1.0f / 16777216.0f);
}

/* Sequential reader over one path's stream: dimension counter + cached block. */
typedef struct {
  uint32_t k0, k1, pixel, sample, dim, blk;
  uint32_t w[4];
} xyzo_stream;

static inline void xyzo_stream_init(xyzo_stream *s, uint64_t seed,
                                    uint32_t pixel, uint32_t sample,
                                    uint32_t dim0) {
  s->k0 = (uint32_t)seed;
  s->k1 = (uint32_t)(seed >> 32);
  s->pixel = pixel;
  s->sample = sample;
  s->dim = dim0;
  s->blk = 0xffffffffu;
}

static inline float xyzo_stream_at(uint64_t seed, uint32_t pixel,
                                   uint32_t sample, uint32_t dim) {
  uint32_t c[4] = {pixel, sample, dim >> 2, 0u}, w[4];
  xyzo_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32), w);
  return xyzo_u01(w[dim & 3]);
}

static inline float xyzo_stream_next(xyzo_stream *s) {
  uint32_t b = s->dim >> 2;
  if (b != s->blk) {
    uint32_t c[4] = {s->pixel, s->sample, b, 0u};
    xyzo_philox4x32_10(c, s->k0, s->k1, s->w);
    s->blk = b;
  }
  float u = xyzo_u01(s->w[s->dim & 3]);
  s->dim++;
  return u;
}
#endif
