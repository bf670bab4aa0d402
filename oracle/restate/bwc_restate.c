/*
 * TEST INFRASTRUCTURE -- not part of the product library; nothing in bigwhoop_b200 links it.
 *
 * Plain-C restatement of the reference codec's hot path (BigWhoop libbwc), written as a
 * straightforward sequential program: per-sample state arrays, the reference's scan order, one
 * MQ coder per codeblock.  It is the CPU oracle that the test suite checks the CUDA kernels
 * against; its own parity with the reference is pinned by golden vectors that the reference
 * library (compiled from its sources) produced, see tests/golden/make_golden.py.
 *
 * Citations are to files of the reference project (src/library/...).
 */
#include "bwc_restate.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef RESTATE_SINGLE
typedef uint32_t rs_raw;
#define PREC_BIT 31
#define MANT_BITS 23
#define EXP_MASK 0x7F800000u
#define MANT_MASK 0x007FFFFFu
#else
typedef uint64_t rs_raw;
#define PREC_BIT 63
#define MANT_BITS 52
#define EXP_MASK 0x7FF0000000000000ull
#define MANT_MASK 0x000FFFFFFFFFFFFFull
#endif
#define SIGN_MASK ((rs_raw)1 << PREC_BIT)

static rs_raw to_raw(rs_float f) {
  rs_raw r;
  memcpy(&r, &f, sizeof r);
  return r;
}

static rs_float from_raw(rs_raw r) {
  rs_float f;
  memcpy(&f, &r, sizeof f);
  return f;
}

int rs_precision_bits(void) { return PREC_BIT; }

/* ---- field normalisation (libbwc.c:622-812, :993-1078, :1093-1176) ------------------------- */

void rs_fill_normalize(const void *src, int src_double, uint64_t n, uint8_t Qm, rs_float *work,
                       rs_float *stats) {
  rs_float mn = 0, mx = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const rs_float v = src_double ? (rs_float)((const double *)src)[i] : (rs_float)((const float *)src)[i];
    work[i] = v;
    if (i == 0 || v > mx) mx = v;
    if (i == 0 || v < mn) mn = v;
  }
  /* parameter_min/max -> alpha, beta (libbwc.c:810-811) */
  const rs_float alpha = (mx + mn) / (rs_float)2.0f;
  const rs_float beta = (rs_float)2.0f / (mx - mn);
  const rs_raw shift = (rs_raw)Qm << MANT_BITS;
  for (uint64_t i = 0; i < n; ++i) {
    rs_float f = (rs_float)(work[i] - alpha) * beta;
    rs_raw r = to_raw(f);
    if ((r & EXP_MASK) != 0 || (r & MANT_MASK) != 0) r += shift;
    work[i] = from_raw(r);
  }
  if (stats) {
    stats[0] = mn;
    stats[1] = mx;
    stats[2] = alpha;
    stats[3] = beta;
  }
}

void rs_denormalize(const rs_float *work, uint64_t n, rs_float pmin, rs_float pmax, uint8_t Qm,
                    void *dst, int dst_double) {
  const rs_float alpha = (pmax + pmin) / (rs_float)2.0f;
  const rs_float beta = (pmax - pmin) / (rs_float)2.0f;
  const rs_raw shift = (rs_raw)Qm << MANT_BITS;
  for (uint64_t i = 0; i < n; ++i) {
    rs_raw r = to_raw(work[i]);
    if ((r & EXP_MASK) != 0 || (r & MANT_MASK) != 0) r -= shift;
    const rs_float f = (rs_float)(from_raw(r) * beta) + alpha;
    if (dst_double)
      ((double *)dst)[i] = (double)f;
    else
      ((float *)dst)[i] = (float)f;
  }
}

/* ---- CDF 9/7 lifting (dwt.c:286-466, :645-789, :1216-2246) ---------------------------------- */

/* lifting coefficients: float literals (dwt.h) widened to the codec's type */
#define L_ALPHA ((rs_float)-1.586134342059924f)
#define L_BETA ((rs_float)-0.052980118572961f)
#define L_GAMMA ((rs_float)0.882911075530934f)
#define L_DELTA ((rs_float)0.360523644801462f)
#define L_KAPPA_H ((rs_float)1.230174104914001f)
#define L_KAPPA_L ((rs_float)0.812893066115961f)
#define EXT 8 /* extension on each side of a line; the lifting reads at most 6 */

/* whole-point symmetric extension of buf[0..len) into buf[-EXT..0) and buf[len..len+EXT),
 * reflecting repeatedly for lines shorter than the extension (dwt.c:286-342) */
static void extend(rs_float *buf, int64_t len) {
  for (int64_t i = 1; i <= EXT; ++i) {
    int64_t j = -i;
    while (j < 0 || j > len - 1) j = (j < 0) ? -j : 2 * (len - 1) - j;
    buf[-i] = buf[j];
    j = len - 1 + i;
    while (j < 0 || j > len - 1) j = (j < 0) ? -j : 2 * (len - 1) - j;
    buf[len - 1 + i] = buf[j];
  }
}

/* dwt.c:354-404 */
static void lift_forward(rs_float *w, int64_t len) {
  for (int64_t i = -3; i < len + 3; i += 2) w[i] += L_ALPHA * (w[i - 1] + w[i + 1]);
  for (int64_t i = -2; i < len + 2; i += 2) w[i] += L_BETA * (w[i - 1] + w[i + 1]);
  for (int64_t i = -1; i < len + 1; i += 2) {
    w[i] += L_GAMMA * (w[i - 1] + w[i + 1]);
    w[i] = L_KAPPA_H * w[i];
  }
  for (int64_t i = 0; i < len; i += 2) {
    w[i] += L_DELTA * (w[i - 1] + w[i + 1]);
    w[i] = L_KAPPA_L * w[i];
  }
}

/* dwt.c:416-466 */
static void lift_inverse(rs_float *w, int64_t len) {
  for (int64_t i = -4; i < len + 4; i += 2) {
    w[i] = L_KAPPA_H * w[i];
    w[i] -= L_DELTA * (w[i - 1] + w[i + 1]);
  }
  for (int64_t i = -5; i < len + 3; i += 2) {
    w[i] = L_KAPPA_L * w[i];
    w[i] -= L_GAMMA * (w[i - 1] + w[i + 1]);
  }
  for (int64_t i = -4; i < len + 2; i += 2) w[i] -= L_BETA * (w[i - 1] + w[i + 1]);
  for (int64_t i = -3; i < len + 1; i += 2) w[i] -= L_ALPHA * (w[i - 1] + w[i + 1]);
}

/* LeGall 5/3 lifting, dwt.c:478-558: the predictor halves the neighbour sum, the update adds
 * (sum + 2) / 4 -- the integer 5/3 rounding offset, applied here in floating point exactly as
 * the reference does */
static void lift_forward_53(rs_float *w, int64_t len) {
  for (int64_t i = -1; i < len + 1; i += 2) w[i] -= (w[i - 1] + w[i + 1]) / 2;
  for (int64_t i = 0; i < len; i += 2) w[i] += (w[i - 1] + w[i + 1] + 2) / 4;
}

static void lift_inverse_53(rs_float *w, int64_t len) {
  for (int64_t i = -2; i < len + 1; i += 2) w[i] -= (w[i - 1] + w[i + 1] + 2) / 4;
  for (int64_t i = -1; i < len; i += 2) w[i] += (w[i - 1] + w[i + 1]) / 2;
}

/* extent of the region transformed at `level` along an axis of n samples with `levels`
 * decompositions: the resolution box ceil((float)n / 2^min(level, levels))
 * (libbwc.c:1539-1548) */
static uint64_t level_extent(uint64_t n, int level, int levels) {
  const int k = level < levels ? level : levels;
  return (uint64_t)ceil((float)n / (float)(1u << k));
}

/* transform every line along axis `a` of the region ext[] (forward: de-interleave lows first,
 * dwt.c:645-721; inverse: interleave first, dwt.c:170-272) */
static void transform_axis(rs_float *work, const uint64_t dims[4], const uint64_t ext[4], int a,
                           int forward, int kernel, rs_float *line) {
  const uint64_t stride[4] = {1, dims[0], dims[0] * dims[1], dims[0] * dims[1] * dims[2]};
  const int64_t len = (int64_t)ext[a];
  const int64_t half = (len + 1) / 2;
  int o[3], k = 0;
  for (int b = 0; b < 4; ++b)
    if (b != a) o[k++] = b;
  rs_float *w = line + EXT;
  for (uint64_t i2 = 0; i2 < ext[o[2]]; ++i2)
    for (uint64_t i1 = 0; i1 < ext[o[1]]; ++i1)
      for (uint64_t i0 = 0; i0 < ext[o[0]]; ++i0) {
        rs_float *base = work + i0 * stride[o[0]] + i1 * stride[o[1]] + i2 * stride[o[2]];
        if (forward) {
          for (int64_t i = 0; i < len; ++i) w[i] = base[i * stride[a]];
          extend(w, len);
          if (kernel == 1) lift_forward_53(w, len); else lift_forward(w, len);
          for (int64_t i = 0; i < len; ++i) {
            const int64_t dst = (i % 2 == 0) ? i / 2 : half + i / 2;
            base[dst * stride[a]] = w[i];
          }
        } else {
          for (int64_t i = 0; i < len; ++i) {
            const int64_t src = (i % 2 == 0) ? i / 2 : half + i / 2;
            w[i] = base[src * stride[a]];
          }
          extend(w, len);
          if (kernel == 1) lift_inverse_53(w, len); else lift_inverse(w, len);
          for (int64_t i = 0; i < len; ++i) base[i * stride[a]] = w[i];
        }
      }
}

static void dwt(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4], int forward,
                const uint8_t kernels[4]) {
  int n_levels = 0;
  for (int a = 0; a < 4; ++a)
    if (decomp[a] > n_levels) n_levels = decomp[a];
  uint64_t maxlen = 1;
  for (int a = 0; a < 4; ++a)
    if (dims[a] > maxlen) maxlen = dims[a];
  rs_float *line = (rs_float *)calloc(maxlen + 2 * EXT, sizeof(rs_float));
  for (int step = 0; step < n_levels; ++step) {
    const int level = forward ? step : n_levels - 1 - step;
    uint64_t ext[4];
    for (int a = 0; a < 4; ++a) ext[a] = level_extent(dims[a], level, decomp[a]);
    for (int q = 0; q < 4; ++q) {
      const int a = forward ? q : 3 - q; /* x, y, z, t forward; t, z, y, x inverse */
      if (level < decomp[a] && ext[a] > 1)
        transform_axis(work, dims, ext, a, forward, kernels[a], line);
    }
  }
  free(line);
}

static const uint8_t CDF97[4] = {0, 0, 0, 0};

void rs_dwt_forward(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4]) {
  dwt(work, dims, decomp, 1, CDF97);
}

void rs_dwt_inverse(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4]) {
  dwt(work, dims, decomp, 0, CDF97);
}

/* Forward transform of one tile's working buffer (dims: the tile's extent; origin: its first
 * sample in field coordinates), dwt.c:1216-1724 with libbwc.c:1539-1548's resolution bounds.
 * A level's region on an axis runs from ceil(origin / 2^k) to ceil((origin + n) / 2^k), k the
 * level capped at the axis's decomposition count.  Where that start is odd (dwt.c:1393-1396)
 * the line's first sample is a high-pass sample: the lifting runs one sample further into the
 * extended buffer, and the flush (dwt.c:645-721) puts the lows w[0], w[2], ... first and the
 * highs w[-1], w[1], ... after them. */
static uint64_t level_bound(uint64_t v, int level, int levels) {
  const int k = level < levels ? level : levels;
  return (uint64_t)ceil((float)v / (float)(1u << k));
}

void rs_dwt_forward_tile(rs_float *work, const uint64_t dims[4], const uint64_t origin[4],
                         const uint8_t decomp[4], const uint8_t kernels[4]) {
  int n_levels = 0;
  uint64_t maxlen = 1;
  for (int a = 0; a < 4; ++a) {
    if (decomp[a] > n_levels) n_levels = decomp[a];
    if (dims[a] > maxlen) maxlen = dims[a];
  }
  rs_float *line = (rs_float *)calloc(maxlen + 2 * EXT + 2, sizeof(rs_float));
  const uint64_t stride[4] = {1, dims[0], dims[0] * dims[1], dims[0] * dims[1] * dims[2]};
  for (int level = 0; level < n_levels; ++level) {
    uint64_t ext[4], r0[4];
    for (int b = 0; b < 4; ++b) {
      r0[b] = level_bound(origin[b], level, decomp[b]);
      ext[b] = level_bound(origin[b] + dims[b], level, decomp[b]) - r0[b];
    }
    for (int a = 0; a < 4; ++a) {
      if (!(level < decomp[a] && ext[a] > 1)) continue;
      const int64_t len = (int64_t)ext[a];
      const int odd = (int)(r0[a] % 2);
      const int64_t half = odd ? len >> 1 : (len + 1) >> 1;
      int o[3], k = 0;
      for (int b = 0; b < 4; ++b)
        if (b != a) o[k++] = b;
      rs_float *B = line + EXT;   /* the line's samples at B[0..len) */
      rs_float *w = B + odd;      /* the lifting's coordinates */
      for (uint64_t i2 = 0; i2 < ext[o[2]]; ++i2)
        for (uint64_t i1 = 0; i1 < ext[o[1]]; ++i1)
          for (uint64_t i0 = 0; i0 < ext[o[0]]; ++i0) {
            rs_float *base = work + i0 * stride[o[0]] + i1 * stride[o[1]] + i2 * stride[o[2]];
            for (int64_t i = 0; i < len; ++i) B[i] = base[i * stride[a]];
            extend(B, len);
            if (kernels[a] == 1) lift_forward_53(w, len); else lift_forward(w, len);
            for (int64_t i = 0; i < half; ++i) base[i * stride[a]] = w[2 * i];
            for (int64_t j = 0; j < len - half; ++j)
              base[(half + j) * stride[a]] = w[2 * j + (odd ? -1 : 1)];
          }
    }
  }
  free(line);
}

/* Inverse transform of one tile's working buffer, dwt.c:1738-2246 with the region bounds of
 * rs_dwt_forward_tile: levels coarsest first, axes t, z, y, x.  fill_inverse_buffer
 * (dwt.c:170-272) puts a line's lows at B[0], B[2], ... and its highs at B[1], B[3], ... whatever
 * the region's start; the buffer is extended like any line; where the start is odd the
 * lifting runs on B + 1, and buffer_flush_inverse (dwt.c:735-789) writes w[-1], w[0], ... =
 * B[0], B[1], ... back in order.
 * Where the start is odd and the length odd, the fill leaves B[len - 1] unwritten (the line's
 * last high lands on B[len], which the extension overwrites) and the reference lifts whatever its
 * per-thread line buffer held there from the previous line, so its output then depends on its
 * OpenMP schedule.  Here that sample is zero, as in a fresh buffer. */
void rs_dwt_inverse_tile(rs_float *work, const uint64_t dims[4], const uint64_t origin[4],
                         const uint8_t decomp[4], const uint8_t kernels[4]) {
  int n_levels = 0;
  uint64_t maxlen = 1;
  for (int a = 0; a < 4; ++a) {
    if (decomp[a] > n_levels) n_levels = decomp[a];
    if (dims[a] > maxlen) maxlen = dims[a];
  }
  rs_float *line = (rs_float *)calloc(maxlen + 2 * EXT + 2, sizeof(rs_float));
  const uint64_t stride[4] = {1, dims[0], dims[0] * dims[1], dims[0] * dims[1] * dims[2]};
  for (int level = n_levels - 1; level >= 0; --level) {
    uint64_t ext[4], r0[4];
    for (int b = 0; b < 4; ++b) {
      r0[b] = level_bound(origin[b], level, decomp[b]);
      ext[b] = level_bound(origin[b] + dims[b], level, decomp[b]) - r0[b];
    }
    for (int a = 3; a >= 0; --a) {
      if (!(level < decomp[a] && ext[a] > 1)) continue;
      const int64_t len = (int64_t)ext[a];
      const int odd = (int)(r0[a] % 2);
      const int64_t half = odd ? len >> 1 : (len + 1) >> 1;
      int o[3], k = 0;
      for (int b = 0; b < 4; ++b)
        if (b != a) o[k++] = b;
      rs_float *B = line + EXT;
      rs_float *w = B + odd;
      for (uint64_t i2 = 0; i2 < ext[o[2]]; ++i2)
        for (uint64_t i1 = 0; i1 < ext[o[1]]; ++i1)
          for (uint64_t i0 = 0; i0 < ext[o[0]]; ++i0) {
            rs_float *base = work + i0 * stride[o[0]] + i1 * stride[o[1]] + i2 * stride[o[2]];
            if (odd && (len & 1)) B[len - 1] = 0;
            for (int64_t i = 0; i < half; ++i) B[2 * i] = base[i * stride[a]];
            for (int64_t i = 0; i < len - half; ++i) B[2 * i + 1] = base[(half + i) * stride[a]];
            extend(B, len);
            if (kernels[a] == 1) lift_inverse_53(w, len); else lift_inverse(w, len);
            for (int64_t i = 0; i < len; ++i) base[i * stride[a]] = B[i];
          }
    }
  }
  free(line);
}

void rs_dwt_forward_kernels(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4],
                            const uint8_t kernels[4]) {
  dwt(work, dims, decomp, 1, kernels);
}

void rs_dwt_inverse_kernels(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4],
                            const uint8_t kernels[4]) {
  dwt(work, dims, decomp, 0, kernels);
}

/* ---- coding tables ------------------------------------------------------------------------ */

/* MQ probability states: the 47-state table of ISO/IEC 15444-1 Table C.2; the reference keeps
 * one copy per MPS sense (mq.c:197-291) */
static const uint16_t QE[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801, 0x3001, 0x2401,
    0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401, 0x3001, 0x2801, 0x2401, 0x2201,
    0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101, 0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1,
    0x0221, 0x0141, 0x0111, 0x0085, 0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
static const uint8_t NMPS[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                                 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
static const uint8_t NLPS[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                                 15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                                 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
static const uint8_t SWITCH[47] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                   0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

/* context labels (mq.h): 9 significance, 1 run, 5 sign, 3 refinement, 1 uniform */
enum { CTX_SIG = 0, CTX_RUN = 9, CTX_SIGN = 10, CTX_MAG = 15, CTX_UNI = 18, CTX_N = 19 };

typedef struct {
  uint8_t state; /* 0..46 */
  uint8_t mps;
} mq_ctx;

static void mq_reset_contexts(mq_ctx *c) {
  /* mq.c:368-375: significance context 0 starts in state 4, run in 3, uniform in 46 */
  for (int i = 0; i < CTX_N; ++i) {
    c[i].state = 0;
    c[i].mps = 0;
  }
  c[CTX_SIG].state = 4;
  c[CTX_RUN].state = 3;
  c[CTX_UNI].state = 46;
}

/* significance context from the neighbour counts h (0-2), v (0-2), d (0-4) for the three
 * subband orientations (tier1.c:231-262) */
static int sig_context(int cls, int h, int v, int d) {
  if (cls == 1) { /* high-pass: horizontal and vertical roles swapped */
    const int t = h;
    h = v;
    v = t;
  }
  if (cls == 2) {
    const int hv = h + v;
    if (d >= 3) return 8;
    if (d == 2) return hv ? 7 : 6;
    if (d == 1) return hv == 0 ? 3 : (hv == 1 ? 4 : 5);
    return hv == 0 ? 0 : (hv == 1 ? 1 : 2);
  }
  if (h == 2) return 8;
  if (h == 1) return v ? 7 : (d ? 6 : 5);
  if (v == 2) return 4;
  if (v == 1) return 3;
  return d >= 2 ? 2 : d;
}

/* sign context and flip bit from the clipped horizontal and vertical sign contributions
 * (-1, 0, +1) (tier1.c:264-275) */
static int sign_context(int h, int v, int *flip) {
  if (h < 0 || (h == 0 && v < 0)) {
    *flip = 1;
    h = -h;
    v = -v;
  } else {
    *flip = 0;
  }
  if (h == 0) return CTX_SIGN + (v != 0 ? 1 : 0);
  return CTX_SIGN + 3 + v; /* h = +1: v -1, 0, +1 -> 2, 3, 4 */
}

/* frac2log (tier1.c:200-216): floor(256 * log2(1 + i / 256)) */
static uint16_t frac2log(unsigned i) { return (uint16_t)floor(256.0 * log2(1.0 + i / 256.0)); }

/* ---- MQ encoder (mq.c:85-127, :328-378, :478-556, :587-759) -------------------------------- */

typedef struct {
  uint32_t A, C, T;
  int32_t t;
  int64_t L;
  uint8_t *b;
  uint64_t cap;
  int overflow;
  mq_ctx ctx[CTX_N];
} mq_enc;

static void put_byte(mq_enc *e) {
  if (e->L >= 0) {
    if ((uint64_t)e->L < e->cap)
      e->b[e->L] = (uint8_t)e->T;
    else
      e->overflow = 1;
  }
  e->L++;
}

static void transfer_byte(mq_enc *e) {
  if (e->T == 0xFF) {
    put_byte(e);
    e->T = (e->C >> 20) & 0xFF;
    e->C &= 0xFFFFF;
    e->t = 7;
    return;
  }
  if (e->C & 0x8000000) {
    e->T++;
    e->C &= 0x7FFFFFF;
  }
  put_byte(e);
  if (e->T == 0xFF) {
    e->T = (e->C >> 20) & 0xFF;
    e->C &= 0xFFFFF;
    e->t = 7;
  } else {
    e->T = (e->C >> 19) & 0xFF;
    e->C &= 0x7FFFF;
    e->t = 8;
  }
}

/* optional record of every coded decision as one byte (context << 1 | decision) and of the
 * decision count at the end of every pass (rs_set_symbol_trace) */
static uint8_t *g_trace;
static uint64_t g_trace_cap, g_trace_n;
static uint64_t *g_trace_pass;

void rs_set_symbol_trace(uint8_t *buf, uint64_t cap, uint64_t *pass_end) {
  g_trace = buf;
  g_trace_cap = cap;
  g_trace_n = 0;
  g_trace_pass = pass_end;
}

uint64_t rs_symbol_trace_count(void) { return g_trace_n; }

static void mq_encode(mq_enc *e, int k, int bit) {
  if (g_trace) {
    if (g_trace_n < g_trace_cap) g_trace[g_trace_n] = (uint8_t)((k << 1) | bit);
    g_trace_n++;
  }
  mq_ctx *c = &e->ctx[k];
  const uint32_t p = QE[c->state];
  e->A -= p;
  if (bit == c->mps) {
    if (e->A & 0x8000) {
      e->C += p;
      return;
    }
    if (e->A < p)
      e->A = p;
    else
      e->C += p;
    c->state = NMPS[c->state];
  } else {
    if (e->A < p)
      e->C += p;
    else
      e->A = p;
    if (SWITCH[c->state]) c->mps ^= 1;
    c->state = NLPS[c->state];
  }
  do {
    e->A <<= 1;
    e->C <<= 1;
    if (--e->t == 0) transfer_byte(e);
  } while (!(e->A & 0x8000));
}

static void mq_flush(mq_enc *e) {
  int n = 12 - e->t;
  e->C <<= e->t;
  while (n > 0) {
    transfer_byte(e);
    n -= e->t;
    e->C <<= e->t;
  }
  transfer_byte(e);
}

typedef struct {
  uint32_t A, C, T;
  int32_t t;
  int64_t L;
} mq_snapshot;

static uint32_t byte_at(const uint8_t *b, uint64_t cap, int64_t i) {
  return (i >= 0 && (uint64_t)i < cap) ? b[i] : 0u;
}

/* minimal truncation length of a pass from the coder state at its end (mq.c:587-675) */
static int64_t truncation_length(const mq_snapshot *s, const uint8_t *b, uint64_t cap) {
  int64_t L = s->L;
#ifdef RESTATE_SINGLE
  int32_t CrFrac = (int32_t)(s->C << s->t);
  int32_t CArFrac = (int32_t)((s->A << s->t) + (uint32_t)CrFrac);
  int32_t CrDec = (int32_t)s->T, CArDec = (int32_t)s->T;
  CrDec += 1 & (CrFrac >> 27);
  CArDec += 1 & (CArFrac >> 27);
  CrFrac &= 0x7FFFFFF;
  CArFrac &= 0x7FFFFFF;
  int sh = 8;
  while (CrDec > 0xFF || CArDec <= 0xFF) {
    const int32_t buff = (int32_t)byte_at(b, cap, L);
    L++;
    CrDec -= buff << (8 - sh);
    CArDec -= buff << (8 - sh);
    CrDec = (int32_t)((uint32_t)CrDec << sh);
    CArDec = (int32_t)((uint32_t)CArDec << sh);
    CrDec += CrFrac >> (27 - sh);
    CArDec += CArFrac >> (27 - sh);
    CrFrac = (int32_t)((uint32_t)CrFrac << sh) & 0x7FFFFFF;
    CArFrac = (int32_t)((uint32_t)CArFrac << sh) & 0x7FFFFFF;
    sh = (buff == 0xFF) ? 7 : 8;
  }
#else
  int64_t Cr = ((int64_t)s->T << 27) + ((int64_t)s->C << s->t);
  int64_t CAr = ((int64_t)s->A << s->t) + Cr;
  int sh = 8;
  while ((Cr >> 27) > 0xFF || (CAr >> 27) <= 0xFF) {
    const int64_t buff = (int64_t)byte_at(b, cap, L);
    L++;
    Cr -= buff << (35 - sh);
    CAr -= buff << (35 - sh);
    Cr = (int64_t)((uint64_t)Cr << sh);
    CAr = (int64_t)((uint64_t)CAr << sh);
    sh = (buff == 0xFF) ? 7 : 8;
  }
#endif
  if (L > 0 && byte_at(b, cap, L - 1) == 0xFF) L--;
  while (L > 1 && byte_at(b, cap, L - 2) == 0xFF && byte_at(b, cap, L - 1) == 0x7F) L -= 2;
  return L;
}

/* ---- codeblock state ------------------------------------------------------------------------ */

typedef struct {
  int W, H, slices;
  uint8_t *sig, *sgn, *visited, *refined, *coded; /* per sample, [slice][y][x] */
  rs_raw *mag;
} cblk_state;

static int st_alloc(cblk_state *s, int W, int H, int slices) {
  const size_t n = (size_t)W * H * slices;
  s->W = W;
  s->H = H;
  s->slices = slices;
  s->sig = (uint8_t *)calloc(n + 1, 1);
  s->sgn = (uint8_t *)calloc(n + 1, 1);
  s->visited = (uint8_t *)calloc(n + 1, 1);
  s->refined = (uint8_t *)calloc(n + 1, 1);
  s->coded = (uint8_t *)calloc(n + 1, 1);
  s->mag = (rs_raw *)calloc(n + 1, sizeof(rs_raw));
  return s->sig && s->sgn && s->visited && s->refined && s->coded && s->mag;
}

static void st_free(cblk_state *s) {
  free(s->sig);
  free(s->sgn);
  free(s->visited);
  free(s->refined);
  free(s->coded);
  free(s->mag);
}

static size_t at(const cblk_state *s, int sl, int y, int x) {
  return ((size_t)sl * s->H + y) * s->W + x;
}

/* significance of neighbour (y + dy, x + dx); rows of the next stripe are only seen from the
 * last row of a full stripe (the reference's causal stripe neighbourhood, tier1.c:692-703) */
static int nb_sig(const cblk_state *s, int sl, int y, int x, int dy, int dx) {
  const int yy = y + dy, xx = x + dx;
  if (yy < 0 || yy >= s->H || xx < 0 || xx >= s->W) return 0;
  if (dy > 0 && (yy >> 2) != (y >> 2) && (y & 3) != 3) return 0;
  return s->sig[at(s, sl, yy, xx)];
}

/* signed contribution of a neighbour: +1 significant positive, -1 significant negative */
static int nb_sign(const cblk_state *s, int sl, int y, int x, int dy, int dx) {
  if (!nb_sig(s, sl, y, x, dy, dx)) return 0;
  return s->sgn[at(s, sl, y + dy, x + dx)] ? -1 : 1;
}

static void neighbour_counts(const cblk_state *s, int sl, int y, int x, int *h, int *v, int *d) {
  *h = nb_sig(s, sl, y, x, 0, -1) + nb_sig(s, sl, y, x, 0, 1);
  *v = nb_sig(s, sl, y, x, -1, 0) + nb_sig(s, sl, y, x, 1, 0);
  *d = nb_sig(s, sl, y, x, -1, -1) + nb_sig(s, sl, y, x, -1, 1) + nb_sig(s, sl, y, x, 1, -1) +
       nb_sig(s, sl, y, x, 1, 1);
}

static int clip1(int v) { return v > 0 ? 1 : (v < 0 ? -1 : 0); }

static int sign_ctx_of(const cblk_state *s, int sl, int y, int x, int *flip) {
  const int h = clip1(nb_sign(s, sl, y, x, 0, -1) + nb_sign(s, sl, y, x, 0, 1));
  const int v = clip1(nb_sign(s, sl, y, x, -1, 0) + nb_sign(s, sl, y, x, 1, 0));
  return sign_context(h, v, flip);
}

/* distortion decrease of a newly significant sample from the five magnitude bits below
 * bit plane b (tier1.c:157-165), and of a refined sample from the six bits below b
 * (tier1.c:139-155) */
static int64_t dist_sig(rs_raw m, int b) {
  int64_t i = 0;
  for (int k = 1; k <= 5; ++k) i = (i << 1) | ((b - k >= 0) ? (int64_t)((m >> (b - k)) & 1) : 0);
  return 49152 + 6144 * i;
}

static int64_t dist_ref(rs_raw m, int b) {
  int64_t i = 0;
  for (int k = 1; k <= 6; ++k) i = (i << 1) | ((b - k >= 0) ? (int64_t)((m >> (b - k)) & 1) : 0);
  return (i < 32) ? 49152 - 2048 * i : 2048 * i - 81920;
}

/* the scan of every pass: slices, then 4-row stripes, then columns, then rows top-down */
#define SCAN(s, ...)                                                                            \
  for (int sl = 0; sl < (s)->slices; ++sl)                                                       \
    for (int y0 = 0; y0 < (s)->H; y0 += 4)                                                       \
      for (int x = 0; x < (s)->W; ++x)                                                           \
        for (int y = y0; y < y0 + 4 && y < (s)->H; ++y) {                                        \
          const size_t i = at((s), sl, y, x);                                                    \
          __VA_ARGS__                                                                            \
        }

/* ---- tier-1 encoder ------------------------------------------------------------------------- */

static uint16_t slope2log(double lambda) {
  /* tier1.c:2100-2130 */
  uint64_t raw;
  memcpy(&raw, &lambda, sizeof raw);
  const uint64_t exponent = ((raw & 0x7FF0000000000000ull) >> 44) - 0x41F00ull;
  const uint64_t mantissa = (raw & 0x000FFFFFFFFFFFFFull) >> 44;
  const uint64_t r = exponent + frac2log((unsigned)mantissa) + 0x10000ull;
  if (r > 0xFFFF) return 0xFFFF;
  if (r < 2) return 2;
  return (uint16_t)r;
}

int rs_context_class(uint32_t hb) {
  /* tier1.c:2416-2446 */
  if ((hb & 3) == 1) return 1;
  if ((hb & 3) == 3) return 2;
  return 0;
}

int64_t rs_t1_encode(const rs_float *work, const uint64_t dims[4], const rs_codeblock *cb,
                     int erres, uint8_t *Kout, uint8_t *Zout, uint64_t *Lout, uint16_t *Sout,
                     uint8_t *bytes, uint64_t cap) {
  const int W = (int)(cb->x1 - cb->x0), H = (int)(cb->y1 - cb->y0);
  const int D = (int)(cb->z1 - cb->z0), T = (int)(cb->t1 - cb->t0);
  cblk_state s;
  if (!st_alloc(&s, W, H, D * T)) {
    st_free(&s);
    return -1;
  }
  /* quantisation (tier1.c:526-729): q = (magnitude / effective step) truncated */
  int K = 0;
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < D; ++z)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          const uint64_t idx = (cb->x0 + x) + dims[0] * ((cb->y0 + y) + dims[1] * ((cb->z0 + z) + dims[2] * (cb->t0 + t)));
          const rs_raw r = to_raw(work[idx]);
          const size_t i = at(&s, z + D * t, y, x);
          s.sgn[i] = (uint8_t)(r >> PREC_BIT);
          const rs_raw q = (rs_raw)(from_raw(r & ~SIGN_MASK) / cb->qt_eff);
          s.mag[i] = q;
          int bl = 0;
          while (bl < PREC_BIT + 1 && (q >> bl)) ++bl;
          if (bl > K) K = bl;
        }
  *Kout = (uint8_t)K;
  if (K == 0) {
    *Zout = 0;
    Sout[0] = 0xFFFF;
    st_free(&s);
    return 0;
  }
  const int Z = 3 * K - 2;
  *Zout = (uint8_t)Z;
  mq_enc e;
  memset(&e, 0, sizeof e);
  e.A = 0x8000;
  e.t = 12;
  e.L = -1;
  e.b = bytes;
  e.cap = cap;
  mq_reset_contexts(e.ctx);
  mq_snapshot snap[RS_MAX_PASSES];
  int64_t dmse[RS_MAX_PASSES];
  int pass = 0;
  for (int b = K - 1; b >= 0; --b) {
    for (int kind = (b == K - 1) ? 2 : 0; kind < 3; ++kind) {
      int64_t mse = 0;
      if (kind == 0) {
        /* significance propagation (tier1.c:962-1146) */
        SCAN(&s, {
          if (s.sig[i]) {
            s.visited[i] = 0;
          } else {
            int h, v, d;
            neighbour_counts(&s, sl, y, x, &h, &v, &d);
            if (h + v + d) {
              const int bit = (int)((s.mag[i] >> b) & 1);
              mq_encode(&e, CTX_SIG + sig_context(cb->cls, h, v, d), bit);
              if (bit) {
                int flip;
                const int k = sign_ctx_of(&s, sl, y, x, &flip);
                mq_encode(&e, k, s.sgn[i] ^ flip);
                mse += dist_sig(s.mag[i], b);
                s.sig[i] = 1;
              }
              s.visited[i] = 1;
            }
          }
        })
      } else if (kind == 1) {
        /* magnitude refinement (tier1.c:1177-1301): samples significant before this bit plane
         * and not coded in its significance propagation pass; the context uses the state
         * before the pass */
        SCAN(&s, { s.coded[i] = s.sig[i] && !s.visited[i]; })
        SCAN(&s, {
          if (s.coded[i]) {
            int k = CTX_MAG;
            if (s.refined[i]) {
              k += 2;
            } else {
              int h, v, d;
              neighbour_counts(&s, sl, y, x, &h, &v, &d);
              /* neighbours refined in this pass were significant already */
              k += (h + v + d) ? 1 : 0;
            }
            mq_encode(&e, k, (int)((s.mag[i] >> b) & 1));
            mse += dist_ref(s.mag[i], b);
            s.refined[i] = 1;
          }
        })
      } else {
        /* cleanup (tier1.c:1332-1511): samples neither significant nor visited; a full
         * stripe column with an empty neighbourhood is coded in run mode */
        for (int sl = 0; sl < s.slices; ++sl)
          for (int y0 = 0; y0 < s.H; y0 += 4)
            for (int x = 0; x < s.W; ++x) {
              int y = y0, run_skip = 0;
              if (y0 + 4 <= s.H) {
                int empty = 1;
                for (int r = 0; r < 4 && empty; ++r) {
                  const size_t i = at(&s, sl, y0 + r, x);
                  int h, v, d;
                  neighbour_counts(&s, sl, y0 + r, x, &h, &v, &d);
                  if (s.sig[i] || s.visited[i] || h + v + d) empty = 0;
                }
                if (empty) {
                  int r = 0;
                  while (r < 4 && !((s.mag[at(&s, sl, y0 + r, x)] >> b) & 1)) ++r;
                  if (r == 4) {
                    mq_encode(&e, CTX_RUN, 0);
                    continue;
                  }
                  mq_encode(&e, CTX_RUN, 1);
                  mq_encode(&e, CTX_UNI, r >> 1);
                  mq_encode(&e, CTX_UNI, r & 1);
                  y = y0 + r;
                  run_skip = 1; /* the first significant row's bit is implied */
                }
              }
              for (; y < y0 + 4 && y < s.H; ++y) {
                const size_t i = at(&s, sl, y, x);
                if (s.sig[i] || s.visited[i]) continue;
                const int bit = (int)((s.mag[i] >> b) & 1);
                if (run_skip) {
                  run_skip = 0;
                } else {
                  int h, v, d;
                  neighbour_counts(&s, sl, y, x, &h, &v, &d);
                  mq_encode(&e, CTX_SIG + sig_context(cb->cls, h, v, d), bit);
                }
                if (bit) {
                  int flip;
                  const int k = sign_ctx_of(&s, sl, y, x, &flip);
                  mq_encode(&e, k, s.sgn[i] ^ flip);
                  mse += dist_sig(s.mag[i], b);
                  s.sig[i] = 1;
                }
              }
            }
        if (erres) {
          /* segmentation symbol 1010 after every bit plane (tier1.c:94-100, :2523-2526) */
          mq_encode(&e, CTX_UNI, 1);
          mq_encode(&e, CTX_UNI, 0);
          mq_encode(&e, CTX_UNI, 1);
          mq_encode(&e, CTX_UNI, 0);
        }
        /* the next bit plane's significance pass starts from scratch */
        SCAN(&s, { s.visited[i] = 0; })
      }
      snap[pass].A = e.A;
      snap[pass].C = e.C;
      snap[pass].T = e.T;
      snap[pass].t = e.t;
      snap[pass].L = e.L;
      dmse[pass] = mse;
      if (g_trace && g_trace_pass) g_trace_pass[pass] = g_trace_n;
      pass++;
    }
  }
  mq_flush(&e);
  const int64_t nbytes = e.L;
  if (e.overflow) {
    st_free(&s);
    return -1;
  }
  /* truncation lengths (mq.c:1151-1175) */
  for (int j = 0; j < Z; ++j) Lout[j] = (uint64_t)truncation_length(&snap[j], bytes, (uint64_t)nbytes);
  /* distortion weights and convex hull (tier1.c:2161-2267, :2477-2531) */
  double mse_d[RS_MAX_PASSES], lambda[RS_MAX_PASSES + 1];
  uint8_t hull[RS_MAX_PASSES + 1];
  double scale = cb->gain_step2 * ldexp(1.0, 2 * K) / 65536.0;
  {
    int j = 0;
    for (int b = K - 1; b >= 0; --b) {
      for (int kind = (b == K - 1) ? 2 : 0; kind < 3; ++kind, ++j) mse_d[j] = (double)dmse[j] * scale;
      scale *= 0.25;
    }
  }
  for (int i = 0; i <= Z; ++i) lambda[i] = 0.0;
  memset(hull, 0, sizeof hull);
  lambda[0] = 18446744073709551616.0;
  int h = 0, hlast = 0;
  for (int i = 0; i < Z; ++i) {
    double dD = 0.0;
    for (int q = hlast; q <= i; ++q) dD += mse_d[q];
    uint64_t dL = (hlast > 0) ? Lout[i] - Lout[hlast - 1] : Lout[i];
    if (dD > 0) {
      while (dD >= lambda[hlast] * (double)dL) {
        lambda[hlast] = 0;
        if (h == 0) break; /* the reference would read below its stack here */
        h--;
        hlast = hull[h];
        dD = 0.0;
        for (int q = hlast; q <= i; ++q) dD += mse_d[q];
        dL = (hlast > 0) ? Lout[i] - Lout[hlast - 1] : Lout[i];
      }
      h++;
      hlast = i + 1;
      hull[h] = (uint8_t)hlast;
      if (dL == 0)
        lambda[hlast] = (dD < 0) ? -1.0 : (dD == 0 ? 0.0 : 18446744073709551616.0);
      else
        lambda[hlast] = dD / (double)dL;
    } else {
      lambda[i + 1] = 0;
    }
  }
  for (int i = 0; i <= Z; ++i) {
    if (lambda[i] < 0)
      Sout[i] = 1;
    else if (lambda[i] == 0)
      Sout[i] = (i == Z) ? 1 : 0;
    else
      Sout[i] = slope2log(lambda[i]);
  }
  st_free(&s);
  return nbytes;
}

/* ---- tier-1 decoder (tier1.c:1543-2069, :2624-2787, :767-931; mq.c:147-173, :846-1029) ---- */

typedef struct {
  uint32_t A, C, T;
  int32_t t;
  int64_t L, Lmax;
  const uint8_t *b;
  mq_ctx ctx[CTX_N];
} mq_dec;

static void fill_lsb(mq_dec *d) {
  if (d->L == d->Lmax || (d->T == 0xFF && d->b[d->L] > 0x8F)) {
    d->t = 8;
    d->C += 0xFF;
  } else if (d->T == 0xFF) {
    d->t = 7;
    d->T = d->b[d->L++];
    d->C += d->T << 1;
  } else {
    d->t = 8;
    d->T = d->b[d->L++];
    d->C += d->T;
  }
}

static void renorm_dec(mq_dec *d) {
  do {
    if (d->t == 0) fill_lsb(d);
    d->A = (d->A << 1) & 0xFFFF;
    d->C <<= 1;
    d->t--;
  } while (!(d->A & 0x8000));
}

static int mq_decode(mq_dec *d, int k) {
  mq_ctx *c = &d->ctx[k];
  const uint32_t p = QE[c->state];
  int x = c->mps;
  d->A = (d->A - p) & 0xFFFF;
  if ((d->C >> 8) >= p) {
    d->C = (d->C - (p << 8)) & 0xFFFFFF;
    if (!(d->A & 0x8000)) {
      if (d->A < p) {
        x = 1 - x;
        if (SWITCH[c->state]) c->mps ^= 1;
        c->state = NLPS[c->state];
      } else {
        c->state = NMPS[c->state];
      }
      renorm_dec(d);
    }
  } else {
    if (d->A < p) {
      c->state = NMPS[c->state];
    } else {
      x = 1 - x;
      if (SWITCH[c->state]) c->mps ^= 1;
      c->state = NLPS[c->state];
    }
    d->A = p;
    renorm_dec(d);
  }
  return x;
}

int rs_t1_decode(rs_float *work, const uint64_t dims[4], const rs_codeblock *cb, int erres,
                 int K, int Z, const uint8_t *data, uint64_t len) {
  const int W = (int)(cb->x1 - cb->x0), H = (int)(cb->y1 - cb->y0);
  const int D = (int)(cb->z1 - cb->z0), T = (int)(cb->t1 - cb->t0);
  cblk_state s;
  if (!st_alloc(&s, W, H, D * T)) {
    st_free(&s);
    return 1;
  }
  int bitplane = 0, cpass = 0;
  if (Z > 0) {
    mq_dec d;
    memset(&d, 0, sizeof d);
    d.b = data;
    d.Lmax = (int64_t)len;
    mq_reset_contexts(d.ctx);
    fill_lsb(&d);
    d.C <<= 8;
    fill_lsb(&d);
    d.C <<= 7;
    d.t -= 7;
    d.A = 0x8000;
    int i = 2, j = Z, k = K, stop = 0;
    while (k-- > 0) {
      const int b = k;
      for (; i < 3; ++i, --j) {
        if (j == 0) {
          stop = 1;
          break;
        }
        if (i == 0) {
          SCAN(&s, {
            if (s.sig[i]) {
              s.visited[i] = 0;
            } else {
              int h, v, dd;
              neighbour_counts(&s, sl, y, x, &h, &v, &dd);
              if (h + v + dd) {
                if (mq_decode(&d, CTX_SIG + sig_context(cb->cls, h, v, dd))) {
                  s.mag[i] |= (rs_raw)1 << b;
                  int flip;
                  const int kk = sign_ctx_of(&s, sl, y, x, &flip);
                  s.sgn[i] = (uint8_t)(mq_decode(&d, kk) ^ flip);
                  s.sig[i] = 1;
                }
                s.visited[i] = 1;
              }
            }
          })
        } else if (i == 1) {
          SCAN(&s, { s.coded[i] = s.sig[i] && !s.visited[i]; })
          SCAN(&s, {
            if (s.coded[i]) {
              int kk = CTX_MAG;
              if (s.refined[i]) {
                kk += 2;
              } else {
                int h, v, dd;
                neighbour_counts(&s, sl, y, x, &h, &v, &dd);
                kk += (h + v + dd) ? 1 : 0;
              }
              if (mq_decode(&d, kk)) s.mag[i] |= (rs_raw)1 << b;
              s.refined[i] = 1;
            }
          })
        } else {
          for (int sl = 0; sl < s.slices; ++sl)
            for (int y0 = 0; y0 < s.H; y0 += 4)
              for (int x = 0; x < s.W; ++x) {
                int y = y0, run_skip = 0;
                if (y0 + 4 <= s.H) {
                  int empty = 1;
                  for (int r = 0; r < 4 && empty; ++r) {
                    const size_t q = at(&s, sl, y0 + r, x);
                    int h, v, dd;
                    neighbour_counts(&s, sl, y0 + r, x, &h, &v, &dd);
                    if (s.sig[q] || s.visited[q] || h + v + dd) empty = 0;
                  }
                  if (empty) {
                    if (!mq_decode(&d, CTX_RUN)) continue;
                    int r = mq_decode(&d, CTX_UNI);
                    r = (r << 1) | mq_decode(&d, CTX_UNI);
                    y = y0 + r;
                    run_skip = 1;
                  }
                }
                for (; y < y0 + 4 && y < s.H; ++y) {
                  const size_t q = at(&s, sl, y, x);
                  if (s.sig[q] || s.visited[q]) continue;
                  int bit;
                  if (run_skip) {
                    run_skip = 0;
                    bit = 1;
                  } else {
                    int h, v, dd;
                    neighbour_counts(&s, sl, y, x, &h, &v, &dd);
                    bit = mq_decode(&d, CTX_SIG + sig_context(cb->cls, h, v, dd));
                  }
                  if (bit) {
                    s.mag[q] |= (rs_raw)1 << b;
                    int flip;
                    const int kk = sign_ctx_of(&s, sl, y, x, &flip);
                    s.sgn[q] = (uint8_t)(mq_decode(&d, kk) ^ flip);
                    s.sig[q] = 1;
                  }
                }
              }
          SCAN(&s, { s.visited[i] = 0; })
        }
      }
      if (stop) break;
      if (erres) {
        int v = mq_decode(&d, CTX_UNI) << 3;
        v |= mq_decode(&d, CTX_UNI) << 2;
        v |= mq_decode(&d, CTX_UNI) << 1;
        v |= mq_decode(&d, CTX_UNI);
        if (v != 0x0A) {
          stop = 1;
          break;
        }
      }
      i = 0;
    }
    if (!stop) i = 0;
    bitplane = (k > 0) ? k : 0;
    cpass = i;
  }
  /* dequantisation (tier1.c:895-910): (m + 0.475 * 2^p) * step with p the first undecoded
   * plane, one higher for samples the interrupted significance pass did not reach */
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < D; ++z)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          const size_t i = at(&s, z + D * t, y, x);
          if (!s.mag[i]) continue;
          const int shift = bitplane + ((!cpass || s.visited[i]) ? 0 : 1);
          rs_float f = (rs_float)s.mag[i];
          f += (float)((uint64_t)1 << shift) * 0.475f;
          f *= cb->qt_eff;
          rs_raw r = to_raw(f) | (s.sgn[i] ? SIGN_MASK : 0);
          work[(cb->x0 + x) + dims[0] * ((cb->y0 + y) + dims[1] * ((cb->z0 + z) + dims[2] * (cb->t0 + t)))] = from_raw(r);
        }
  st_free(&s);
  return 0;
}
