/*
 * TEST INFRASTRUCTURE -- not part of the product library.
 *
 * Plain-C restatement of the reference codec's hot path (BigWhoop libbwc), used by the test
 * suite as an independent CPU oracle for the CUDA kernels: field normalisation, the CDF 9/7
 * lifting transform, EBCOT tier-1 encoding with the MQ coder (truncation lengths and
 * convex-hull slopes included) and tier-1 decoding with dequantisation.
 *
 * Parity of this restatement is pinned by golden vectors produced with the reference library
 * itself (compiled from its sources; see tests/golden/make_golden.py).
 *
 * Compiled twice: the default build restates the reference's double-precision build
 * (bwc_float = double, 63 magnitude bits); -DRESTATE_SINGLE restates its single-precision build.
 */
#ifndef BWC_RESTATE_H
#define BWC_RESTATE_H

#include <stdint.h>

#ifdef RESTATE_SINGLE
typedef float rs_float;
#else
typedef double rs_float;
#endif

#define RS_MAX_PASSES 190

#ifdef __cplusplus
extern "C" {
#endif

/* magnitude bits of a quantised sample (63 or 31) */
int rs_precision_bits(void);

/* fill_buffer + normalize_param (libbwc.c:622-812, :993-1078): copies n samples of `src`
 * (double when src_double, else float) into `work`, finds min/max, applies
 * f = (f - alpha) * beta with alpha = (max + min) / 2, beta = 2 / (max - min), then adds Qm to
 * the exponent of every non-zero sample.  stats = {min, max, alpha, beta}. */
void rs_fill_normalize(const void *src, int src_double, uint64_t n, uint8_t Qm, rs_float *work,
                       rs_float *stats);

/* denormalize_param + flush (libbwc.c:1093-1176, :827-978) */
void rs_denormalize(const rs_float *work, uint64_t n, rs_float pmin, rs_float pmax, uint8_t Qm,
                    void *dst, int dst_double);

/* forward / inverse multi-level 9/7 transform of a (nX, nY, nZ, nTS) buffer, x fastest, with
 * decomp[a] levels along axis a (dwt.c:1216-1724, :1738-2246) */
void rs_dwt_forward(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4]);
void rs_dwt_inverse(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4]);
/* the same with a wavelet kernel per axis: 0 CDF 9/7, 1 LeGall 5/3 (dwt.c:478-558; the Haar
 * kernel is not restated: the reference has no boundary extension for it, dwt.c:1259-1262) */
void rs_dwt_forward_kernels(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4],
                            const uint8_t kernels[4]);
void rs_dwt_inverse_kernels(rs_float *work, const uint64_t dims[4], const uint8_t decomp[4],
                            const uint8_t kernels[4]);
/* forward transform of one tile of a multi-tile field: dims = the tile's extent, origin = its
 * first sample in field coordinates (odd region starts follow dwt.c:1393-1396, 645-721) */
void rs_dwt_forward_tile(rs_float *work, const uint64_t dims[4], const uint64_t origin[4],
                         const uint8_t decomp[4], const uint8_t kernels[4]);

/* its inverse (the reference's odd-start inverse: lows at B[0], B[2], ..., lifting on B + 1) */
void rs_dwt_inverse_tile(rs_float *work, const uint64_t dims[4], const uint64_t origin[4],
                         const uint8_t decomp[4], const uint8_t kernels[4]);

/* one codeblock: box in working-buffer coordinates and its subband's coding parameters */
typedef struct {
  uint64_t x0, y0, z0, t0;
  uint64_t x1, y1, z1, t1;
  rs_float qt_eff;       /* qt_effective_step_size */
  double gain_step2;     /* (double)dwt_gain * (double)(qt_step_size^2 in rs_float) */
  int cls;               /* significance-context class: 0 low-pass, 1 high-pass, 2 diagonal */
} rs_codeblock;

/* significance-context class of a subband from its highband flag (bit 0 x, 1 y, 2 z, 3 t) */
int rs_context_class(uint32_t highband_flag);

/* encode_codeblock (tier1.c:2303-2588): K, Z, truncation lengths L[0..Z), log slopes
 * S[0..Z], coded bytes (at most cap).  Returns the number of coded bytes produced by the
 * terminated MQ codeword, or -1 when cap is too small. */
int64_t rs_t1_encode(const rs_float *work, const uint64_t dims[4], const rs_codeblock *cb,
                     int erres, uint8_t *K, uint8_t *Z, uint64_t *L, uint16_t *S, uint8_t *bytes,
                     uint64_t cap);

/* Records, during the following rs_t1_encode calls, every coded decision as one byte
 * (context << 1 | decision) into buf (up to cap) and the running decision count at the end of
 * every pass into pass_end[pass]; buf = NULL stops recording.  rs_symbol_trace_count returns
 * the number of decisions seen since the last rs_set_symbol_trace. */
void rs_set_symbol_trace(uint8_t *buf, uint64_t cap, uint64_t *pass_end);
uint64_t rs_symbol_trace_count(void);

/* decode_codeblock + cblkcopy_inverse (tier1.c:2624-2787, :767-931): decodes Z passes of a
 * codeblock with K significant bit planes from len bytes and writes the dequantised samples
 * into `work` (whose codeblock region must be zero).  Returns 0. */
int rs_t1_decode(rs_float *work, const uint64_t dims[4], const rs_codeblock *cb, int erres,
                 int K, int Z, const uint8_t *data, uint64_t len);

#ifdef __cplusplus
}
#endif

#endif
