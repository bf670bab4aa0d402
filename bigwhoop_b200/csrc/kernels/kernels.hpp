// Host-visible interface of the CUDA kernels (plain C++; no CUDA types besides cudaStream_t).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "../host/common.hpp"

namespace bwcb {

// One codeblock as the tier-1 kernels see it.
struct CbDev {
  uint32_t x0, y0, z0, t0;   // origin in the parameter's working buffer
  uint32_t w, h, d, nt;      // extents along x, y, z, t
  uint64_t out_off;          // byte offset of the codeblock's coded bytes
  uint64_t scratch_off;      // compress: byte offset of its bit planes;
                             // decompress: element offset of its magnitudes
  uint32_t out_cap;          // compress: capacity of the coded-byte region
  uint32_t sb;               // index into the SbDev table
  uint64_t base;             // element offset of the codeblock's field in the working buffer
  uint64_t sy, sz, st;       // that field's strides along y, z and t (elements)
  uint32_t slot;             // which slope-range pair (min, max) the codeblock updates
  uint32_t pad;
};

// One subband.
struct SbDev {
  double gain_step2;   // (double)dwt_gain * (double)(qt_step_size * qt_step_size)
  bwc_float qt_eff;    // qt_effective_step_size
  uint32_t Kmax;
  uint32_t cls;        // significance-context class: 0 low-pass, 1 high-pass, 2 diagonal
  uint32_t erres;      // error resilience of the field (segmentation symbols after each plane)
  uint32_t pad;
};

// Outputs and scratch of the tier-1 encoder.
struct T1EncOut {
  uint8_t *bytes;        // coded bytes, codeblock c at CbDev::out_off
  uint8_t *K;            // [ncb]
  uint8_t *Z;            // [ncb]
  uint32_t *L;           // [ncb * kMaxPasses] truncation lengths
  uint16_t *S;           // [ncb * (kMaxPasses + 1)] log slopes
  uint32_t *slopes;      // [2 * slots]: per slot min over non-zero slopes, max (atomics;
                         //   init 0xFFFF / 0); CbDev::slot selects the pair
  uint32_t *flags;       // [ncb]: 1 coded-byte overflow, 2 hull stack underflow,
                         //        4 unsettled truncation scan, 8 symbol arena full
  uint8_t *planes;       // scratch: bit planes, CbDev::scratch_off
  uint64_t *snaps;       // scratch: [ncb * kMaxPasses * 2] end-of-pass coder states
  int64_t *dmse;         // scratch: [ncb * kMaxPasses] distortion decrease per pass
  uint8_t *symbols;      // scratch: symbol arena
  uint64_t sym_cap;      //   its capacity in bytes
  unsigned long long *sym_used;   // [0] bump counter of the arena (bytes reserved), [1] decisions
                                  // coded (both zeroed by the caller)
  uint32_t *pass_count;  // scratch: [ncb * kMaxPasses] symbols per pass
  uint64_t *pass_off;    // scratch: [ncb * kMaxPasses] arena offset of each pass's symbols
};

struct FieldDims {
  uint64_t width, height, depth, dt;
};

// field.cu
// A box of w x h x d x t samples of a field: element (x, y, z, t) at base + x + sy*y + sz*z +
// st*t (the tiles of a multi-tile field).
struct BoxMap {
  uint64_t w, h, d;
  uint64_t base, sy, sz, st;
};
void launch_fill_minmax_box(const void *src, bool src_double, uint64_t n, const BoxMap &m,
                            bwc_float *work, uint64_t *keys, cudaStream_t s);
void launch_denormalize_box(const bwc_float *work, uint64_t n, bwc_float pmin, bwc_float pmax,
                            uint8_t Qm, void *dst, bool dst_double, const BoxMap &m,
                            cudaStream_t s);
void launch_fill_minmax(const void *src, bool src_double, uint64_t n, bwc_float *work,
                        uint64_t *minmax_keys, cudaStream_t s);
void launch_normalize(bwc_float *work, uint64_t n, const uint64_t *minmax_keys, uint8_t Qm,
                      bwc_float *stats_out, cudaStream_t s);
void launch_denormalize(const bwc_float *work, uint64_t n, bwc_float pmin, bwc_float pmax,
                        uint8_t Qm, void *dst, bool dst_double, cudaStream_t s);

// dwt.cu: the multi-level separable transform (CDF 9/7 or LeGall 5/3 per axis) of one parameter.
// level_ext[l] = extents (x, y, z, t) of the region transformed at level l; axis_on[l] bit a
// set when axis a is transformed at level l.
// kern[a]: the axis's wavelet kernel, 0 CDF 9/7, 1 LeGall 5/3; odd[l] bit a: the level's region
// starts at an odd coordinate along axis a (tiles of a multi-tile field).
struct DwtPlan {
  int levels;
  uint64_t ext[16][4];
  uint8_t axis_on[16];
  uint8_t kern[4];
  uint8_t odd[16];
};
// Forward: `temp` holds the normalised field on entry, the coefficients end in `work`;
// inverse: `temp` holds the coefficients, the field ends in `work`.  `temp` is scratch after.
void launch_dwt_forward(bwc_float *work, bwc_float *temp, const FieldDims &dims,
                        const DwtPlan &plan, cudaStream_t s);
void launch_dwt_inverse(bwc_float *work, bwc_float *temp, const FieldDims &dims,
                        const DwtPlan &plan, cudaStream_t s);
// copies the transform's fault word (non-zero: a bulk-copy batch never arrived and the
// coefficients are incomplete) to `host` (page-locked) on `s` and clears it
void dwt_fault_download(uint32_t *host, cudaStream_t s);
// looks up the fault word of the current device (call before capturing transforms in a graph)
void dwt_setup();

// t1_encode.cu: context modelling (one CTA per codeblock, max_cols = largest number of stripe
// columns of a codeblock) followed by MQ coding (one thread per codeblock).
size_t t1_model_smem(uint32_t max_cols);
// scratch bytes (bit planes) of one codeblock of ncols stripe columns
uint64_t t1_scratch_bytes(uint64_t ncols);
// Each codeblock addresses its samples as work[base + x + y*sy + z*sz + t*st].  `order`
// (optional, device) lists the codeblocks largest first: the MQ kernel's lanes take them in
// that order, and with `queue` (one device counter per phase, room for eight, zeroed here) the
// modelling kernel runs persistent and takes codeblocks from that work queue.  With an order, a
// queue and at least 2048 codeblocks, the order is modelled in four phases on `s` (one CTA per
// codeblock, in order) and each phase's MQ kernel runs on a side stream once its phase is
// modelled; `s` waits for them before it goes on.
// `after_model` (optional) is recorded on `s` after the (last) modelling launch; `mq_times`
// (optional) receives the MQ launches' start and end events.
// Timing events (created by the caller, timing enabled) that launch_t1_encode records around
// each MQ launch, on the stream that launch runs on; `n` is set to the number of launches.
struct T1LaunchTimes {
  cudaEvent_t start[8] = {}, end[8] = {};
  int n = 0;
};
void launch_t1_encode(const bwc_float *work, const CbDev *cbs, uint32_t ncb, const SbDev *sbs,
                      const T1EncOut &out, uint32_t max_cols, cudaStream_t s,
                      const uint32_t *order = nullptr, uint32_t *queue = nullptr,
                      cudaEvent_t after_model = nullptr, T1LaunchTimes *mq_times = nullptr);

// t1_decode.cu: decodes Z[c] passes of codeblock c from data + out_off (Lmax[c] bytes) and
// writes the dequantised samples into the (zeroed) working buffer.
// Codeblocks of up to 4096 stripe columns (max_cols) decode through the mask-based decoder,
// larger ones through the column-state decoder (state_cap / gstate / grid apply to it only).
// mags: decode scratch, t1_decode_scratch_elems(ncols) elements per codeblock at scratch_off.
void launch_t1_decode_ex(bwc_float *work, const CbDev *cbs, uint32_t ncb,
                         const SbDev *sbs, const uint8_t *data, const uint8_t *K,
                         const uint8_t *Z, const uint32_t *Lmax, uchar erres, bwc_raw *mags,
                         uint32_t *flags, uint32_t state_cap, uint16_t *gstate,
                         uint32_t *work_counter, int grid, cudaStream_t s,
                         const uint32_t *order, uint32_t max_cols);
uint64_t t1_decode_scratch_elems(uint64_t ncols);

// mlp.cu: the rate-control warm start's network (34 -> 64 -> 64 -> 1, FP32).
constexpr int kMlpInputs = kRateFeatures;
constexpr int kMlpParams = 64 * kMlpInputs + 64 + 64 * 64 + 64 + 64 + 1;
// predictions for n (<= 64) feature rows with the model set by bwc_b200_set_rate_model;
// false when no model is set
bool mlp_predict(const float *features, int n, float *out);

// gather.cu: dst[p.dst .. +size) = (p.from_blob ? blob : dev)[p.src .. +size)
void launch_gather(uint8_t *dst, const uint8_t *blob, const uint8_t *dev,
                   const GatherPiece *pieces, uint64_t npieces, cudaStream_t s);

}  // namespace bwcb
