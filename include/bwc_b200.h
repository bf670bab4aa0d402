/*
 * bwc_b200.h -- additional entry points of the B200 BigWhoop library.
 *
 * None of these has a counterpart in the reference API; they are additive exports beside the
 * drop-in bwc.h interface.  Existing bwc_* signatures are unchanged.
 *
 * Device-resident buffers: bwc_compress and bwc_decompress accept CUDA device pointers as
 * well as host pointers for stream->inp and stream->out (the pointer kind is queried with
 * cudaPointerGetAttributes); device-resident input skips the host-to-device copy, a
 * device-resident output receives the result by a device-to-device copy.
 */
#ifndef BWC_B200_H
#define BWC_B200_H

#include "bwc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Library identification: returns PREC_BIT of the loaded library (63 double, 31 single). */
int bwc_b200_precision_bits(void);

/* The reference keeps process-wide subband energy gains that every configure_codec and
 * bwc_set_decomp call adds to (dwt.c:80, :808-1066); codestreams depend on that history.
 * reset returns the table to its load-time state; get copies its 3 x 10 doubles. */
void bwc_b200_reset_gain_state(void);
void bwc_b200_get_gain_state(double *out30);

/* Intermediate results of the next bwc_compress on `codec` (parameter 0 of tile 0), copied to
 * host memory when the pointer is non-NULL:
 *   normalized, transformed : the working buffer (tile-size bwc_float values) after
 *                             normalisation and after the wavelet transform;
 *   K, Z                    : per codeblock, in tier-1 order;
 *   L                       : per codeblock MAXIMUM_NO_PASSES truncation lengths;
 *   S                       : per codeblock MAXIMUM_NO_PASSES + 1 log slopes;
 *   bytes / byte_offsets    : coded bytes of every codeblock (L[Z-1] each), packed in
 *                             tier-1 order, and each codeblock's start in `bytes`;
 *   stats                   : min, max, alpha, beta of parameter 0 (bwc_float).
 * Capacities are the caller's: normalized/transformed hold the tile size, the per-codeblock
 * arrays hold bwc_b200_num_codeblocks(codec, 0) entries, bytes holds bytes_cap bytes. */
typedef struct
{
  bwc_float *normalized;
  bwc_float *transformed;
  uint8     *K;
  uint8     *Z;
  uint32    *L;
  uint16    *S;
  uint8     *bytes;
  uint64     bytes_cap;
  uint64    *byte_offsets;
  bwc_float *stats;
  uint32    *flags;
} bwc_b200_stage_dump;

uint64 bwc_b200_num_codeblocks(bwc_codec *const codec, uint8 const param);
void   bwc_b200_set_stage_dump(bwc_codec *const codec, bwc_b200_stage_dump const *dump);

/* Decompression counterpart: the working buffer after tier-1 decoding (dequantised
 * coefficients) and after the inverse transform, parameter 0 of tile 0. */
typedef struct
{
  bwc_float *dequantized;
  bwc_float *reconstructed;
} bwc_b200_decode_dump;

void   bwc_b200_set_decode_dump(bwc_codec *const codec, bwc_b200_decode_dump const *dump);

/* Host-only inspection (no samples are coded by these).
 * codeblock_geometry: X0,Y0,Z0,TS0,X1,Y1,Z1,TS1 of codeblock c (tier-1 order) in the
 *   parameter's working buffer, its subband's high-pass flags and Kmax;
 * subband_steps: effective quantisation step, step size and energy gain of its subband;
 * parsed_codeblock: after bwc_create_decompression, K (= Kmax - Kmsbs), Kmsbs, Z and the
 *   MAXIMUM_NO_PASSES truncation lengths recovered from the packet headers;
 * assemble_from_tier1: runs rate control, packet formation and codestream layout of a codec
 *   prepared by bwc_create_compression on caller-supplied tier-1 results (all parameters'
 *   codeblocks in tier-1 order; L and S strided by MAXIMUM_NO_PASSES and MAXIMUM_NO_PASSES + 1;
 *   coded bytes at byte_offsets[c] of `bytes`; minmax = min, max per parameter) and writes the
 *   codestream to stream->out.  Returns its size, 0 on error. */
int    bwc_b200_codeblock_geometry(bwc_codec *const codec, uint8 const param, uint64 const c,
                                   uint64 *geom10);
int    bwc_b200_subband_steps(bwc_codec *const codec, uint8 const param, uint64 const c,
                              double *out3);
int    bwc_b200_parsed_codeblock(bwc_codec *const codec, uint8 const param, uint64 const c,
                                 int64 *meta3, uint64 *L);
/* the same for codeblock c of parameter `param` in tile `tile` of a multi-tile codestream
 * (bwc_create_decompression parses those).  No
 * counterpart in the reference. */
int    bwc_b200_parsed_codeblock_of_tile(bwc_codec *const codec, uint32 const tile,
                                         uint8 const param, uint64 const c, int64 *meta3,
                                         uint64 *L);
size_t bwc_b200_assemble_from_tier1(bwc_codec *const codec, bwc_stream *const stream,
                                    uint8 const *K, uint8 const *Z, uint64 const *L,
                                    uint16 const *S, uint8 const *bytes,
                                    uint64 const *byte_offsets, bwc_float const *minmax,
                                    uint16 const slope_min, uint16 const slope_max);
/* The same for a codec of one or more tiles (bwc_set_tiles): codeblocks of every tile in tile
 * order, within a tile parameter by parameter; minmax = min, max per tile and parameter;
 * slopes = slope minimum, maximum per tile.  This runs the host half of multi-tile coding
 * alone (per-tile rate control, packets, the multi-tile codestream), on tier-1 results made
 * elsewhere.  No counterpart in the reference. */
size_t bwc_b200_assemble_tiles_from_tier1(bwc_codec *const codec, bwc_stream *const stream,
                                          uint8 const *K, uint8 const *Z, uint64 const *L,
                                          uint16 const *S, uint8 const *bytes,
                                          uint64 const *byte_offsets, bwc_float const *minmax,
                                          uint16 const *slopes);

/* Device time of the stages of the last bwc_compress / bwc_decompress on this codec, in
 * milliseconds (CUDA events on the codec's stream): [0] upload, [1] fill+normalise, [2] wavelet,
 * [3] tier-1, [4] download of tier-1 results, [5] tier-2 (host), [6] codestream gather and
 * download, [7] total, [8] tier-1 symbols coded (millions, compression), [9] tier-1 context
 * modelling (compression: from the start of tier-1 to the end of its last modelling launch),
 * [10] the MQ coder launches' device time, summed over launches (compression; the launches run
 * on side streams and overlap the modelling of later codeblocks, so [9] + [10] can exceed [3]),
 * [11] the number of those launches.  Returns the number of entries written (at most n). */
int    bwc_b200_last_timings(bwc_codec *const codec, double *out_ms, int n);

/* Batched compression of n independently configured codecs (each set up with
 * bwc_create_compression as for bwc_compress, with its own stream).  No counterpart in the
 * reference API.  Every codestream is byte-identical to what bwc_compress would produce for that
 * codec; sizes[i] receives its length (0 on failure).  The fields' transforms run concurrently,
 * tier-1 codes all their codeblocks in one pass, tier-2 runs in parallel host threads and one
 * device gather assembles every codestream.  Returns 0 on success, 1 on failure.  One batch runs
 * at a time per device (calls are serialised). */
uchar  bwc_b200_compress_batch(bwc_codec *const *codecs, bwc_stream *const *streams, uint32 n,
                               size_t *sizes);

/* Stage times (ms) of the last batch on the current device: [0] set-up and uploads,
 * [1] fill/normalise/transform, [2] tier-1, [3] tier-2 (host), [4] gather and outputs,
 * [5] whole call; then the counts [6] of CUDA graphs captured and [7] of graph launches so far
 * (the fill/normalise/transform phase runs as a graph, captured once per batch signature).
 * Returns the number of entries written (at most n). */
int    bwc_b200_last_batch_timings(double *out_ms, int n);

/* Codeblocks per warp the MQ coder uses for a launch of `ncb` codeblocks on the current GPU:
 * the autotuned value when this GPU model has tuned that size class (its first tier-1 launch of
 * the class times the candidates; BWC_B200_TUNE_FILE persists results, BWC_B200_AUTOTUNE=0
 * disables tuning), else the built-in rule.  No counterpart in the reference API. */
int    bwc_b200_mq_lanes(uint32 ncb);

/* Forward transform path for the levels that transform x, y and z: mode 0 = the 3D tile kernel
 * only; 1 (default) = the TMA z-streaming kernel wherever x, y and z span at least 8 and rows
 * start on 16-byte boundaries (even widths in FP64, multiples of 4 in FP32), else the register
 * z-streaming kernel where x and y span at least 48 samples and the level gives every SM at
 * least 8 plane pairs, else the tile kernel; 2 = as 1, with the register z-streaming kernel
 * wherever x, y and z span at least 8; 3 = the register z-streaming kernel wherever x, y and z
 * span at least 8, never the TMA one.  ctas > 0 fixes the streaming kernels' grids (their CTAs
 * split the level's units evenly), 0 = one CTA per SM.  Process-wide; set it between calls.
 * All settings give bit-identical coefficients.  No counterpart in the reference API. */
void   bwc_b200_set_transform_tuning(int mode, int ctas);

/* Rate-control warm start.  No counterpart in the reference API.
 *
 * The reference's rate control bisects, per quality layer, over a 16-bit log-slope threshold;
 * every probe depends on the previous one.  With a model set, the library predicts each layer's
 * final threshold with a small network (34 -> 64 -> 64 -> 1, ReLU, FP32; hand-written CUDA
 * kernels), evaluates the whole probe path that prediction implies at once (in parallel host
 * threads) and replays the exact bisection over those results; a path that leaves the predicted
 * one costs another round.  The probes, their order and the selected thresholds are the plain
 * search's, so the codestream is byte-identical with or without a model.
 *
 * Network parameters: BWC_B200_MLP_PARAMS floats, W1[64][34], b1[64], W2[64][64], b2[64],
 * W3[64], b3.  Inputs (bwc_b200_rate_features): a 32-bin histogram of the codeblocks' non-zero
 * pass slopes (bins of 2048), log(layer bits per value) / 4, (log(values) - 14) / 4.  Output:
 * final threshold / 65536.
 *
 * set_rate_model     : copies the parameters (NULL: plain bisection); process-wide.  Until it
 *                      is called, the library uses its built-in model (trained by
 *                      bigwhoop_b200/ratemodel.py on 2000 synthetic fields).
 * rate_features      : the 34 inputs of `layer` in the last compression of `codec`.
 * rate_stats         : of that layer: final threshold, probes, rounds of dependent probes,
 *                      predicted threshold (-1 without a model), slope range min and max.
 * mlp_forward        : y[n] = network(X[n][34]) (host arrays; runs on the current device).
 * mlp_gradient       : gradient of mean((y - t)^2) over the n rows, and that loss.
 * mlp_train          : `epochs` passes of Adam (learning rate lr, minibatches of `batch` rows
 *                      drawn in a seeded order) starting from and updating `params`; the mean
 *                      minibatch loss of every epoch goes to loss_per_epoch (may be NULL).
 * All return 0 on success. */
#define BWC_B200_MLP_PARAMS 6465
int    bwc_b200_set_rate_model(const float *params);
int    bwc_b200_rate_features(bwc_codec *const codec, uint8 const layer, float *out34);
int    bwc_b200_rate_stats(bwc_codec *const codec, uint8 const layer, double *out6);
int    bwc_b200_mlp_forward(const float *params, const float *X, uint32 n, float *y);
int    bwc_b200_mlp_gradient(const float *params, const float *X, const float *t, uint32 n,
                             float *grad, float *loss);
int    bwc_b200_mlp_train(float *params, const float *X, const float *t, uint32 n,
                          uint32 epochs, uint32 batch, float lr, uint64 seed,
                          float *loss_per_epoch);

/* Tier-1 encoding of ONE codeblock without any memory allocation.  No counterpart in the
 * reference API.
 *
 * For callers that cannot call cudaMalloc -- code that gets its device memory from a
 * framework's pool, latency-bound services that cannot take the synchronisation an
 * allocation implies.  The caller passes device buffers it owns; the library's own working
 * memory (bit planes, symbol arena, coder snapshots) is one fixed static device area of about
 * 2.9 MB (double build; 1.5 MB single), held by every GPU that loads the library until the
 * process exits.
 *
 *   coeffs          device pointer: wavelet coefficients of one parameter, nX x nY x nZ x nTS
 *                   bwc_float values, x fastest (the layout bwc_compress transforms into);
 *   box             host array: X0, Y0, Z0, TS0, X1, Y1, Z1, TS1 of the codeblock in `coeffs`;
 *   qt_eff          the subband's effective quantisation step;
 *   gain_step2      (double)dwt_gain * (double)(qt_step_size * qt_step_size), the distortion
 *                   weight of the subband;
 *   highband        the subband's high-pass axis flags (bit 0 x, 1 y, 2 z, 3 t);
 *   erres           error resilience (segmentation symbols);
 *   K, Z            device, one byte each: significant bit planes and coding passes;
 *   L, S            device: MAXIMUM_NO_PASSES truncation lengths and MAXIMUM_NO_PASSES + 1
 *                   log slopes (only the first Z, resp. Z + 1, are written);
 *   bytes           device: the codeblock's coded bytes, bytes_cap of room (L[Z-1] are
 *                   valid; up to 16 zero bytes after them are written too);
 *   status          device, one uint32: 0, or 1 = bytes_cap too small, 2/4 = see the flags of
 *                   the stage dump (not expected), 8 = symbol arena full (not possible within
 *                   the size limit), 16 = symbol staging overflow (not possible);
 *   stream          cudaStream_t to run on (NULL = default stream).
 * Results are identical to what bwc_compress computes for the same codeblock.
 *
 * Limit: at most 4096 stripe columns (width x ceil(height / 4) x depth x time steps, e.g. a
 * 32 x 32 x 16 codeblock); larger ones are rejected with a message on stderr and return 1.
 * Returns 0 once the work is queued on `stream`, 1 on rejected arguments or a CUDA error (an
 * error already pending from the caller's earlier CUDA calls is refused before anything is
 * queued).  `stream` must belong to the current device on every call.
 *
 * The static area is shared by every call on a device and keeps the last call's contents (each
 * call clears what must start at zero), so calls that overlap on the GPU (different streams, or
 * host threads without ordering) race and corrupt each other; order them on one stream.  The
 * first call on a device looks up the area's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture. */
int    bwc_b200_t1_encode_codeblock_static(const bwc_float *coeffs, uint64 nX, uint64 nY,
                                           uint64 nZ, uint64 nTS, const uint64 *box,
                                           bwc_float qt_eff, double gain_step2, uint8 highband,
                                           uchar erres, uint8 *K, uint8 *Z, uint32 *L,
                                           uint16 *S, uint8 *bytes, uint32 bytes_cap,
                                           uint32 *status, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BWC_B200_H */
