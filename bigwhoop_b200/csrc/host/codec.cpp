// Codec configuration, setters and geometry (the host half of the libbwc API).
//
// Behavioural contract: every setter and derived quantity here reproduces the reference's
// observable state bit for bit -- the control fields callers read, the step sizes, Kmax and
// energy gains that shape the codestream, and the float-rounded tile/resolution/subband/
// precinct/codeblock boxes (libbwc.c:161-607, :1345-1716, :1828-2828, dwt.c:808-1202).  The
// arithmetic is written out with the reference's own operand types (float divisions inside
// double ceil/floor, uint32 wrap-around in codeblock offsets) because those roundings decide
// where codeblock boundaries fall.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "common.hpp"

namespace bwcb {

const char *kMemError =
    "o##########################################################o\n"
    "|                   ERROR: Out of memory                   |\n"
    "o##########################################################o\n";
const char *kCsError =
    "o##########################################################o\n"
    "|                ERROR: Invalid Codestream                 |\n"
    "o##########################################################o\n";

void warn(const char *msg) { fputs(msg, stderr); }

// ---------------------------------------------------------------------------------------------
// Wavelet energy gains.
//
// The reference keeps the subband energy gains in one process-wide table that every call of
// initialize_gain_lut (from configure_codec and bwc_set_decomp, dwt.c:808-1066) ADDS to
// instead of overwriting: after n calls each entry holds the n-fold running sum.  The gains
// enter the rate-distortion slopes of every codeblock, so codestreams depend on how many codecs
// the process has configured before.  This table reproduces that state exactly: the same sums,
// accumulated term by term in the same order into a process-global table.
// ---------------------------------------------------------------------------------------------
namespace {
constexpr int kMaxDecompLevels = 4;   // dwt.h:69
double g_gain[3][2 * kMaxDecompLevels + 2];
std::mutex g_gain_mutex;

// filter taps as the reference stores them: float literals widened to double (dwt.h:77-116)
const double kTaps97[2][5] = {
    {(double)-0.091271763114250f, (double)-0.057543526228500f, (double)0.591271763114250f,
     (double)1.115087052457000f, 0.0},
    {(double)0.053497514821620f, (double)0.033728236885750f, (double)-0.156446533057980f,
     (double)-0.533728236885750f, (double)1.205898036472721f}};
const double kTaps53[2][5] = {{(double)0.5f, (double)1.0f, 0, 0, 0},
                              {(double)-0.125f, (double)-0.25f, (double)0.75f, 0, 0}};
const double kTapsHaar[2][5] = {{1.0, 1.0, 0, 0, 0}, {-0.5, 0.5, 0, 0, 0}};

// Symmetric (odd-length) filters: square norm of the filter iterated `levels` times through
// the low-pass branch, accumulated into lut[0..3] (dwt.c:875-970).
void accumulate_symmetric(double *lut_row, const double (*taps)[5], int len_lo, int len_hi,
                          double *b1, double *b2) {
  const int lfb = len_lo;
  double *lut = lut_row + 1;
  int lgb = len_lo;
  for (int j = 0; j < 2; ++j) {
    for (int k = 0; k < lgb + 1; ++k) b1[k] = b1[2 * lgb - k] = taps[j][k];
    for (int k = 0; k < 2 * lgb + 1; ++k) lut[0] += b1[k] * b1[k];
    for (int k = 1; k < kMaxDecompLevels; ++k) {
      for (int l = 0; l < 2 * lgb + 1; ++l) {
        b2[2 * l + lfb] += b1[l] * taps[0][lfb];
        for (int m = 0; m < lfb; ++m) {
          b2[2 * l + m] += b1[l] * taps[0][m];
          b2[2 * l + (2 * lfb - m)] += b1[l] * taps[0][m];
        }
      }
      double *t = b1; b1 = b2; b2 = t;
      std::memset(b2, 0, 512 * sizeof(double));
      lgb = 2 * lgb + lfb;
      for (int l = 0; l < 2 * lgb + 1; ++l) lut[k] += b1[l] * b1[l];
    }
    lut += kMaxDecompLevels + 1;
    lgb = len_hi;
  }
  std::memset(b1, 0, 512 * sizeof(double));
  std::memset(b2, 0, 512 * sizeof(double));
}

// Haar (even-length) branch (dwt.c:976-1059).
void accumulate_haar(double *lut_row, double *b1, double *b2) {
  const int lfb = 2;
  double *lut = lut_row + 1;
  int lgb = 2;
  for (int j = 0; j < 2; ++j) {
    for (int k = 0; k < lgb; ++k) b1[k] = kTapsHaar[j][k];
    for (int k = 0; k < lgb; ++k) lut[0] += b1[k] * b1[k];
    for (int k = 1; k < kMaxDecompLevels; ++k) {
      for (int l = 0; l < lgb; ++l)
        for (int m = 0; m < lfb; ++m) b2[2 * l + m] += b1[l] * kTapsHaar[0][m];
      double *t = b1; b1 = b2; b2 = t;
      std::memset(b2, 0, 512 * sizeof(double));
      lgb = lgb * lfb;
      for (int l = 0; l < lgb; ++l) lut[k] += b1[l] * b1[l];
    }
    lut += kMaxDecompLevels + 1;
    lgb = 2;
  }
}
}  // namespace

uchar initialize_gain_lut() {
  std::lock_guard<std::mutex> lock(g_gain_mutex);
  std::vector<double> a(512, 0.0), b(512, 0.0);
  for (int f = 0; f < 3; ++f) g_gain[f][0] = g_gain[f][kMaxDecompLevels + 1] = 1.0;
  accumulate_symmetric(g_gain[bwc_dwt_9_7], kTaps97, 3, 4, a.data(), b.data());
  accumulate_symmetric(g_gain[bwc_dwt_5_3], kTaps53, 1, 2, a.data(), b.data());
  accumulate_haar(g_gain[bwc_dwt_haar], a.data(), b.data());
  return 0;
}

void reset_gain_lut() {
  std::lock_guard<std::mutex> lock(g_gain_mutex);
  std::memset(g_gain, 0, sizeof(g_gain));
}

void copy_gain_lut(double *out30) {
  std::lock_guard<std::mutex> lock(g_gain_mutex);
  std::memcpy(out30, g_gain, sizeof(g_gain));
}

// get_dwt_energy_gain (dwt.c:1082-1202): product over the transformed axes.
bwc_float dwt_energy_gain(const bwc_gl_ctrl &c, uchar hb, uint16_t level) {
  std::lock_guard<std::mutex> lock(g_gain_mutex);
  const uint8_t dec[4] = {c.decompX, c.decompY, c.decompZ, c.decompTS};
  const int kern[4] = {(int)c.KernelX, (int)c.KernelY, (int)c.KernelZ, (int)c.KernelTS};
  double Gb = 1.0;
  for (int a = 0; a < 4; ++a) {
    int8_t lv = (int8_t)((level > dec[a]) ? dec[a] : level);
    if (lv != 0) {
      while (lv > kMaxDecompLevels) { Gb *= 2.0; lv--; }
      Gb *= g_gain[kern[a]][lv + ((hb >> a) & 1) * (kMaxDecompLevels + 1)];
    }
  }
  return (bwc_float)Gb;
}

// Derived quantisation (libbwc.c:1957-1979 with bwc_float, :2392-2414 with double): the
// exponent/mantissa of the base step delta = 1/(2^(2+PREC_BIT) * sqrt(G)).
template <typename T>
static void derive_step(bwc_gl_ctrl *c, T delta) {
  for (c->qt_exponent = 0; delta < 1; ++c->qt_exponent, delta *= 2) {
  }
  c->qt_mantissa = (uint16_t)std::floor(0.5f + ((delta - 1.0f) * (1 << 16)));
  if (c->qt_exponent > (uint32_t)kPrecBit) {
    c->qt_exponent = kPrecBit;
    c->qt_mantissa = 0;
  }
  if (c->qt_mantissa >= 1u << 16) {
    if (c->qt_exponent == 0) {
      c->qt_mantissa = (1 << 16) - 1;
    } else {
      c->qt_exponent--;
      c->qt_mantissa = 0;
    }
  }
}

}  // namespace bwcb

using namespace bwcb;

// ---------------------------------------------------------------------------------------------
// Public API: allocation and configuration
// ---------------------------------------------------------------------------------------------
static bwc_codec *alloc_codec() {
  bwc_codec *codec = (bwc_codec *)calloc(1, sizeof(bwc_codec));
  if (!codec) {
    warn(kMemError);
    return nullptr;
  }
  codec->info.codec_prec = (kPrecByte == 8) ? bwc_precision_double : bwc_precision_single;
  return codec;
}

namespace bwcb {
bool unsupported_kernel(const bwc_gl_ctrl &c, const bwc_gl_inf &info) {
  const int kern[4] = {(int)c.KernelX, (int)c.KernelY, (int)c.KernelZ, (int)c.KernelTS};
  const uint8_t dec[4] = {c.decompX, c.decompY, c.decompZ, c.decompTS};
  const uint64_t n[4] = {info.nX, info.nY, info.nZ, info.nTS};
  for (int a = 0; a < 4; ++a)
    if (dec[a] > 0 && n[a] > 1 && kern[a] != bwc_dwt_9_7 && kern[a] != bwc_dwt_5_3) return true;
  return false;
}
}  // namespace bwcb

extern "C" bwc_stream *bwc_init_stream(void *const inpbuf, void *const outbuf, bwc_mode const mode) {
  bwc_stream *s = (bwc_stream *)calloc(1, sizeof(bwc_stream));
  if (!s) {
    warn(kMemError);
    return nullptr;
  }
  s->inp = inpbuf;
  s->out = outbuf;
  s->mode = mode;
  return s;
}

static uchar set_span(bwc_span **slot, const char *src, uint64_t size) {
  *slot = (bwc_span *)calloc(1, sizeof(bwc_span));
  if (!*slot) {
    warn(kMemError);
    return 1;
  }
  (*slot)->memory = (uchar *)calloc(size ? size : 1, 1);
  if (!(*slot)->memory) {
    warn(kMemError);
    return 1;
  }
  std::memcpy((*slot)->memory, src, size);
  (*slot)->access = (*slot)->memory;
  (*slot)->size = size;
  (*slot)->position = 0;
  return 0;
}

extern "C" uchar bwc_set_com(bwc_stream *const data, char const *const com, uint16 const size) {
  return set_span(&data->codestream.com, com, size);
}

extern "C" uchar bwc_set_aux(bwc_stream *const data, char const *const aux, uint32 const size) {
  return set_span(&data->codestream.aux, aux, size);
}

extern "C" bwc_codec *configure_codec(bwc_codec *const codec, uint64 const nX, uint64 const nY,
                                      uint64 const nZ, uint64 const nTS, uint8 const nPar,
                                      bwc_precision const prec) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  info->nX = nX; info->nY = nY; info->nZ = nZ; info->nTS = nTS;
  info->nPar = nPar;
  info->data_prec = prec;

  c->tileSizeX = nX; c->tileSizeY = nY; c->tileSizeZ = nZ; c->tileSizeTS = nTS;
  c->nTiles = 1;
  c->precSizeX = (nX >> 1) ? 15 : 0;
  c->precSizeY = (nY >> 1) ? 15 : 0;
  c->precSizeZ = (nZ >> 1) ? 15 : 0;
  c->precSizeTS = (nTS >> 1) ? 15 : 0;
  c->cbX = (nX >> 1) ? 5 : 0;
  c->cbY = (nY >> 1) ? 5 : 0;
  c->cbZ = (nZ >> 1) ? 5 : 0;
  c->cbTS = (nTS >> 1) ? 5 : 0;
  c->KernelX = c->KernelY = c->KernelZ = c->KernelTS = bwc_dwt_9_7;
  c->progression = bwc_prog_LRCP;
  c->quantization_style = bwc_qt_derived;
  c->nLayers = 0;
  c->Qm = kPrecBit - 1;
  c->bitrate = nullptr;
  c->guard_bits = 2;

  // (uint8)(log(n)/log(2)) exactly as libbwc.c:1920-1923 computes it
  uint8_t lx = (uint8_t)(std::log((double)nX) / std::log(2.0));
  uint8_t ly = (uint8_t)(std::log((double)nY) / std::log(2.0));
  uint8_t lz = (uint8_t)(std::log((double)nZ) / std::log(2.0));
  uint8_t lt = (uint8_t)(std::log((double)nTS) / std::log(2.0));
  c->decompX = (nX >> 1) ? ((4 < lx) ? 4 : lx) : 0;
  c->decompY = (nY >> 1) ? ((4 < ly) ? 4 : ly) : 0;
  c->decompZ = (nZ >> 1) ? ((4 < lz) ? 4 : lz) : 0;
  c->decompTS = (nTS >> 1) ? ((4 < lt) ? 4 : lt) : 0;
  c->nDecomp = std::max(c->decompX, std::max(c->decompY, std::max(c->decompZ, c->decompTS)));

  if (initialize_gain_lut()) {
    bwc_free_codec(codec);
    return nullptr;
  }
  bwc_float delta = (bwc_float)(1 / (std::pow(2, 2 + kPrecBit) *
                                     std::sqrt((double)dwt_energy_gain(*c, 0, c->nDecomp))));
  derive_step<bwc_float>(c, delta);
  return codec;
}

extern "C" bwc_codec *bwc_alloc_coder(uint64 const nX, uint64 const nY, uint64 const nZ,
                                      uint64 const nTS, uint8 const nPar,
                                      bwc_precision const prec) {
  bwc_codec *codec = alloc_codec();
  if (!codec) return nullptr;
  codec = configure_codec(codec, nX, nY, nZ, nTS, nPar, prec);
  if (codec) codec->mode = comp;
  return codec;
}

extern "C" bwc_codec *bwc_alloc_decoder(void) {
  bwc_codec *codec = alloc_codec();
  if (codec) codec->mode = decomp;
  return codec;
}

extern "C" void bwc_free_codec(bwc_codec *const codec) {
  if (!codec) return;
  free_engine(codec);
  free(codec->control.bitrate);
  free(codec);
}

extern "C" void bwc_set_error_resilience(bwc_codec *const codec) {
  codec->control.error_resilience ^= 0x01;
  codec->control.CSsgc ^= (0x01 << 0);
}

extern "C" void set_quant_style(bwc_codec *const codec, bwc_quant_st const style) {
  codec->control.quantization_style = style;
  codec->control.CSsgc |= (0x01 << 1);
}

extern "C" void set_quant_step_size(bwc_codec *const codec, double const delta_in) {
  if ((delta_in <= 0) || (delta_in >= 2)) {
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
         "   WARNING: Invalid quantization step size                    \n"
         "                                                              \n"
         "            The quantization step size does not lie within    \n"
         "            the acceptable range of:                          \n"
         "                                                              \n"
         "                          0 < step size < 2                   \n"
         ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n");
    return;
  }
  derive_step<double>(&codec->control, delta_in);
  codec->control.CSsgc |= (0x01 << 2);
}

extern "C" void set_progression(bwc_codec *const codec, bwc_prog_ord const progression) {
  codec->control.progression = progression;
  codec->control.CSsgc |= (0x01 << 3);
}

extern "C" void set_kernels(bwc_codec *const codec, bwc_dwt_filter const KernelX,
                            bwc_dwt_filter const KernelY, bwc_dwt_filter const KernelZ,
                            bwc_dwt_filter const KernelTS) {
  bwc_gl_ctrl *c = &codec->control;
  // a zero argument selects the default filter; for the time axis that default is Haar
  c->KernelX = KernelX ? KernelX : bwc_dwt_9_7;
  c->KernelY = KernelY ? KernelY : bwc_dwt_9_7;
  c->KernelZ = KernelZ ? KernelZ : bwc_dwt_9_7;
  c->KernelTS = KernelTS ? KernelTS : bwc_dwt_haar;
  c->CSsgc |= (0x01 << 4);
}

extern "C" void bwc_set_decomp(bwc_codec *const codec, uint8 const dX, uint8 const dY,
                               uint8 const dZ, uint8 const dTS) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  uint8_t lx = (uint8_t)(std::log((double)info->nX) / std::log(2.0));
  uint8_t ly = (uint8_t)(std::log((double)info->nY) / std::log(2.0));
  uint8_t lz = (uint8_t)(std::log((double)info->nZ) / std::log(2.0));
  uint8_t lt = (uint8_t)(std::log((double)info->nTS) / std::log(2.0));
  c->decompX = (info->nX >> 1) ? ((dX < lx) ? dX : lx) : 0;
  c->decompY = (info->nY >> 1) ? ((dY < ly) ? dY : ly) : 0;
  c->decompZ = (info->nZ >> 1) ? ((dZ < lz) ? dZ : lz) : 0;
  c->decompTS = (info->nTS >> 1) ? ((dTS < lt) ? dTS : lt) : 0;
  c->nDecomp = std::max(c->decompX, std::max(c->decompY, std::max(c->decompZ, c->decompTS)));
  if ((c->decompX > 63) || (c->decompY > 63) || (c->decompZ > 63) || (c->decompTS > 31)) {
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
         "   WARNING: Invalid decomposition level value                 \n"
         "                                                              \n"
         "            The maximum acceptable decomposition level is     \n"
         "            63 for all spatial and 31 for the temporal        \n"
         "            dimensions.                                       \n"
         ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n");
    c->decompX = (info->nX >> 1) ? 4 : 0;
    c->decompY = (info->nY >> 1) ? 4 : 0;
    c->decompZ = (info->nZ >> 1) ? 4 : 0;
    c->decompTS = (info->nTS >> 1) ? 4 : 0;
    return;
  }
  if (initialize_gain_lut()) {
    bwc_free_codec(codec);
    return;
  }
  double delta = 1 / (std::pow(2, 2 + kPrecBit) *
                      std::sqrt((double)dwt_energy_gain(*c, 0, c->nDecomp)));
  derive_step<double>(c, delta);
  c->CSsgc |= (0x01 << 5);
}

extern "C" void bwc_set_precincts(bwc_codec *const codec, uint8 const pX, uint8 const pY,
                                  uint8 const pZ, uint8 const pTS) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  c->precSizeX = (info->nX >> 1) ? (pX ? pX : 15) : 0;
  c->precSizeY = (info->nY >> 1) ? (pY ? pY : 15) : 0;
  c->precSizeZ = (info->nZ >> 1) ? (pZ ? pZ : 15) : 0;
  c->precSizeTS = (info->nTS >> 1) ? (pTS ? pTS : 15) : 0;
  if (((c->precSizeX < 1) && (info->nX >> 1)) || ((c->precSizeY < 1) && (info->nY >> 1)) ||
      ((c->precSizeZ < 1) && (info->nZ >> 1)) || ((c->precSizeTS < 1) && (info->nTS >> 1)) ||
      (c->precSizeX > 15) || (c->precSizeY > 15) || (c->precSizeZ > 15) || (c->precSizeTS > 15)) {
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
         "   WARNING: Invalid precinct size                             \n"
         "                                                              \n"
         "            The maximum acceptable precinct size is 2^15,     \n"
         "            the smallest valid precinct size is 2^1.          \n"
         ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n");
    c->precSizeX = (info->nX >> 1) ? 15 : 0;
    c->precSizeY = (info->nY >> 1) ? 15 : 0;
    c->precSizeZ = (info->nZ >> 1) ? 15 : 0;
    c->precSizeTS = (info->nTS >> 1) ? 15 : 0;
    return;
  }
  c->CSsgc |= (0x01 << 6);
}

extern "C" void bwc_set_codeblocks(bwc_codec *const codec, uint8 const cbX, uint8 const cbY,
                                   uint8 const cbZ, uint8 const cbTS) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  c->cbX = (info->nX >> 1) ? (cbX ? cbX : 5) : 0;
  c->cbY = (info->nY >> 1) ? (cbY ? cbY : 5) : 0;
  c->cbZ = (info->nZ >> 1) ? (cbZ ? cbZ : 5) : 0;
  c->cbTS = (info->nTS >> 1) ? (cbTS ? cbTS : 5) : 0;
  int sum = c->cbX + c->cbY + c->cbZ + c->cbTS;
  if ((c->cbX > 10) || (c->cbY > 10) || (c->cbZ > 10) || (c->cbTS > 10) || sum < 4 || sum > 20) {
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
         "   WARNING: Invalid codeblock size                            \n"
         "                                                              \n"
         "            The maximum acceptable codeblock size is 2^20     \n"
         "            with a maximum allowable number of datapoints     \n"
         "            in each dimension of 2^10. The smallest valid     \n"
         "            codeblock size is 2^4.                            \n"
         ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n");
    c->cbX = (info->nX >> 1) ? 5 : 0;
    c->cbY = (info->nY >> 1) ? 5 : 0;
    c->cbZ = (info->nZ >> 1) ? 5 : 0;
    c->cbTS = (info->nTS >> 1) ? 5 : 0;
    return;
  }
  c->CSsgc |= (0x01 << 7);
}

extern "C" void bwc_set_qm(bwc_codec *const codec, uint8 const Qm) {
  if ((int8_t)(kPrecBit - Qm) < 1) {
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
         "   WARNING: Invalid Q number formate range                    \n"
         "                                                              \n"
         "            The specified Q number formate range is larger    \n");
    warn(kPrecBit == 31 ? "            than the permitted 30 bits.                       \n"
                        : "            than the permitted 62 bits.                       \n");
    warn(">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n");
    return;
  }
  codec->control.Qm = Qm;
  codec->control.CSsgc |= (0x01 << 8);
}

static uint64_t ceil_ratio_f(uint64_t a, uint64_t b) {
  // ceil(((float)a / b)): float division, then ceil in double (libbwc.c:2717-2720)
  return (uint64_t)std::ceil((double)((float)a / (float)b));
}

extern "C" void bwc_set_tiles(bwc_codec *const codec, uint64 const tX, uint64 const tY,
                              uint64 const tZ, uint64 const tTS, bwc_tile_instr const instr) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  const char *dims_warn =
      ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n"
      "   WARNING: Invalid Tile Dimensions                           \n"
      "                                                              \n"
      "            One or more of the specified tile dimensions      \n"
      "            has a value that falls outside of its valid       \n"
      "            range. Please verify that all tile dimension      \n"
      "            are within the range of:                          \n"
      "                                                              \n"
      "                 16 ≤ Tile_Size_Xi ≤ Grid_Points_Xi           \n"
      ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>><<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n";
  auto bad = [&]() {
    return (c->tileSizeX < 16 && c->tileSizeX > info->nX) ||
           (c->tileSizeY < 16 && c->tileSizeY > info->nY) ||
           (c->tileSizeZ < 16 && c->tileSizeZ > info->nZ) ||
           (c->tileSizeTS < 16 && c->tileSizeTS > info->nTS);
  };
  if (instr == bwc_tile_sizeof) {
    if (bad()) {
      warn(dims_warn);
      return;
    }
    c->tileSizeX = (info->nX >> 1) ? (tX ? tX : info->nX) : info->nX;
    c->tileSizeY = (info->nY >> 1) ? (tY ? tY : info->nY) : info->nY;
    c->tileSizeZ = (info->nZ >> 1) ? (tZ ? tZ : info->nZ) : info->nZ;
    c->tileSizeTS = (info->nTS >> 1) ? (tTS ? tTS : info->nTS) : info->nTS;
  } else {
    c->tileSizeX = (info->nX >> 1) ? (tX ? ceil_ratio_f(info->nX, tX) : info->nX) : info->nX;
    c->tileSizeY = (info->nY >> 1) ? (tY ? ceil_ratio_f(info->nY, tY) : info->nY) : info->nY;
    c->tileSizeZ = (info->nZ >> 1) ? (tZ ? ceil_ratio_f(info->nZ, tZ) : info->nZ) : info->nZ;
    c->tileSizeTS = (info->nTS >> 1) ? (tTS ? ceil_ratio_f(info->nTS, tTS) : info->nTS) : info->nTS;
    if (bad()) {
      warn(dims_warn);
      c->tileSizeX = info->nX; c->tileSizeY = info->nY;
      c->tileSizeZ = info->nZ; c->tileSizeTS = info->nTS;
      return;
    }
  }
  c->nTiles = ceil_ratio_f(info->nX, c->tileSizeX) * ceil_ratio_f(info->nY, c->tileSizeY) *
              ceil_ratio_f(info->nZ, c->tileSizeZ) * ceil_ratio_f(info->nTS, c->tileSizeTS);
  c->CSsgc |= (0x01 << 9);
}

// ---------------------------------------------------------------------------------------------
// Geometry (create_codec, libbwc.c:1345-1716)
// ---------------------------------------------------------------------------------------------
namespace bwcb {

static uint8_t popcount4(uint8_t v) {   // subband_gain, libbwc.c:319-343
  uint8_t t = v;
  t -= (t >> 1) & 0x55;
  t = (t & 0x33) + ((t >> 2) & 0x33);
  return (t + (t >> 4)) & 0x0F;
}

// (uint16)((a0 == a1) ? 0 : ceil((float)a1 / s - floor((float)a0 / s)))
static uint16_t count_cells(uint64_t a0, uint64_t a1, uint64_t s) {
  if (a0 == a1) return 0;
  double v = std::ceil((double)((float)a1 / (float)s) - std::floor((double)((float)a0 / (float)s)));
  return (uint16_t)v;
}

static uint64_t res_bound(uint64_t v, int shift) {   // (uint64)ceil((float)v / (1 << shift))
  return (uint64_t)std::ceil((double)((float)v / (float)(1 << shift)));
}

static uint64_t sub_bound(uint64_t v, int shift, int high) {
  // (uint64)ceil(((float)v / (1 << shift)) - 0.5 * high)
  return (uint64_t)std::ceil((double)((float)v / (float)(1 << shift)) - 0.5 * high);
}

static uint32_t prec_halve(uint32_t v, int high) {   // (uint32)ceil(((float)v / 2) - 0.5 * high)
  return (uint32_t)std::ceil((double)((float)v / 2.0f) - 0.5 * high);
}

static uchar init_precinct(const bwc_gl_ctrl &c, Parameter &par, Precinct &pr, uint32_t dX,
                           uint32_t dY, uint32_t dZ, uint32_t dTS, uint32_t sb_index,
                           uint32_t prec_index) {
  const uint64_t csX = 1ull << c.cbX, csY = 1ull << c.cbY, csZ = 1ull << c.cbZ, csT = 1ull << c.cbTS;
  pr.numCbX = count_cells(pr.X0, pr.X1, csX);
  pr.numCbY = count_cells(pr.Y0, pr.Y1, csY);
  pr.numCbZ = count_cells(pr.Z0, pr.Z1, csZ);
  pr.numCbTS = count_cells(pr.TS0, pr.TS1, csT);
  pr.ncb = (uint64_t)pr.numCbX * pr.numCbY * pr.numCbZ * pr.numCbTS;
  pr.first_cb = par.codeblocks.size();
  if (!pr.ncb) return 0;
  tagtree_init(pr.msbs, pr.numCbX, pr.numCbY, pr.numCbZ, pr.numCbTS);
  tagtree_init(pr.incl, pr.numCbX, pr.numCbY, pr.numCbZ, pr.numCbTS);
  if (pr.msbs.nodes.empty() || pr.incl.nodes.empty()) return 1;
  const uint32_t fX = (uint32_t)std::floor((double)((float)pr.X0 / (float)csX));
  const uint32_t fY = (uint32_t)std::floor((double)((float)pr.Y0 / (float)csY));
  const uint32_t fZ = (uint32_t)std::floor((double)((float)pr.Z0 / (float)csZ));
  const uint32_t fT = (uint32_t)std::floor((double)((float)pr.TS0 / (float)csT));
  uint32_t idx = 0;
  for (uint16_t t = 0; t < pr.numCbTS; ++t)
    for (uint16_t z = 0; z < pr.numCbZ; ++z)
      for (uint16_t y = 0; y < pr.numCbY; ++y)
        for (uint16_t x = 0; x < pr.numCbX; ++x, ++idx) {
          Codeblock cb;
          cb.subband = sb_index;
          cb.precinct = prec_index;
          cb.idx = idx;
          // dX + (uint32)MAX(...): 32-bit wrap-around as in libbwc.c:292-299
          cb.box.X0 = (uint32_t)(dX + (uint32_t)std::max<uint64_t>(pr.X0, csX * (uint32_t)(x + fX)));
          cb.box.Y0 = (uint32_t)(dY + (uint32_t)std::max<uint64_t>(pr.Y0, csY * (uint32_t)(y + fY)));
          cb.box.Z0 = (uint32_t)(dZ + (uint32_t)std::max<uint64_t>(pr.Z0, csZ * (uint32_t)(z + fZ)));
          cb.box.TS0 = (uint32_t)(dTS + (uint32_t)std::max<uint64_t>(pr.TS0, csT * (uint32_t)(t + fT)));
          cb.box.X1 = (uint32_t)(dX + (uint32_t)std::min<uint64_t>(pr.X1, csX * (uint32_t)(x + fX + 1)));
          cb.box.Y1 = (uint32_t)(dY + (uint32_t)std::min<uint64_t>(pr.Y1, csY * (uint32_t)(y + fY + 1)));
          cb.box.Z1 = (uint32_t)(dZ + (uint32_t)std::min<uint64_t>(pr.Z1, csZ * (uint32_t)(z + fZ + 1)));
          cb.box.TS1 = (uint32_t)(dTS + (uint32_t)std::min<uint64_t>(pr.TS1, csT * (uint32_t)(t + fT + 1)));
          par.codeblocks.push_back(std::move(cb));
        }
  return 0;
}

static uchar init_subband(bwc_codec *codec, Parameter &par, uint32_t r, uint8_t hb) {
  const bwc_gl_ctrl &c = codec->control;
  Resolution &res = par.res[r];
  Subband sb;
  const int decomp_level = c.nDecomp - (int)r + 1;
  const int lX = (decomp_level > c.decompX) ? c.decompX : decomp_level;
  const int lY = (decomp_level > c.decompY) ? c.decompY : decomp_level;
  const int lZ = (decomp_level > c.decompZ) ? c.decompZ : decomp_level;
  const int lT = (decomp_level > c.decompTS) ? c.decompTS : decomp_level;
  sb.box.X0 = sub_bound(par.box.X0, lX, (hb & kDimX) ? 1 : 0);
  sb.box.Y0 = sub_bound(par.box.Y0, lY, (hb & kDimY) ? 1 : 0);
  sb.box.Z0 = sub_bound(par.box.Z0, lZ, (hb & kDimZ) ? 1 : 0);
  sb.box.TS0 = sub_bound(par.box.TS0, lT, (hb & kDimTS) ? 1 : 0);
  sb.box.X1 = sub_bound(par.box.X1, lX, (hb & kDimX) ? 1 : 0);
  sb.box.Y1 = sub_bound(par.box.Y1, lY, (hb & kDimY) ? 1 : 0);
  sb.box.Z1 = sub_bound(par.box.Z1, lZ, (hb & kDimZ) ? 1 : 0);
  sb.box.TS1 = sub_bound(par.box.TS1, lT, (hb & kDimTS) ? 1 : 0);

  const uint32_t Rb = kPrecBit + popcount4(hb);
  sb.highband = hb;
  sb.dwt_gain = dwt_energy_gain(c, hb, (uint16_t)decomp_level);
  if (c.quantization_style == bwc_qt_none) {
    sb.qt_exponent = (uint8_t)Rb;
    sb.qt_mantissa = 0;
    sb.qt_step = 1;
    sb.qt_eff = 1;
  } else {
    sb.qt_exponent = (uint8_t)(c.qt_exponent + ((r == 0) ? 0 : 1 - (int)r));
    sb.qt_mantissa = (uint16_t)c.qt_mantissa;
    sb.qt_step = (bwc_float)((1.0f + ((double)sb.qt_mantissa / (1 << 11))) / std::pow(2, sb.qt_exponent));
    sb.qt_eff = (bwc_float)(1.0f + ((double)sb.qt_mantissa / (1 << 11)));
    if (sb.qt_exponent > Rb)
      sb.qt_eff = (bwc_float)(sb.qt_eff / std::pow(2, sb.qt_exponent - Rb));
    else
      sb.qt_eff = (bwc_float)(sb.qt_eff * std::pow(2, Rb - sb.qt_exponent));
  }
  sb.Kmax = (uint16_t)std::max(0, (int)c.guard_bits + (int)sb.qt_exponent - 1);

  const uint64_t pX = 1ull << c.precSizeX, pY = 1ull << c.precSizeY;
  const uint64_t pZ = 1ull << c.precSizeZ, pT = 1ull << c.precSizeTS;
  uint64_t sbsX = 0, sbsY = 0, sbsZ = 0, sbsT = 0;
  if (r > 0) {
    const Box &lo = par.res[r - 1].box;
    sbsX = (hb & kDimX) ? lo.X1 - lo.X0 : 0;
    sbsY = (hb & kDimY) ? lo.Y1 - lo.Y0 : 0;
    sbsZ = (hb & kDimZ) ? lo.Z1 - lo.Z0 : 0;
    sbsT = (hb & kDimTS) ? lo.TS1 - lo.TS0 : 0;
  }
  const uint32_t sb_index = (uint32_t)par.subbands.size();
  sb.first_precinct = (uint32_t)par.precincts.size();
  par.subbands.push_back(sb);

  if (!res.nprec) return 0;
  const Box &rb = res.box;
  for (uint16_t pt = 0; pt < res.numPTS; ++pt)
    for (uint16_t pz = 0; pz < res.numPZ; ++pz)
      for (uint16_t py = 0; py < res.numPY; ++py)
        for (uint16_t px = 0; px < res.numPX; ++px) {
          Precinct pr;
          pr.X0 = (uint32_t)std::max<uint64_t>(rb.X0, pX * (uint32_t)(px + (uint32_t)(rb.X0 / pX)));
          pr.Y0 = (uint32_t)std::max<uint64_t>(rb.Y0, pY * (uint32_t)(py + (uint32_t)(rb.Y0 / pY)));
          pr.Z0 = (uint32_t)std::max<uint64_t>(rb.Z0, pZ * (uint32_t)(pz + (uint32_t)(rb.Z0 / pZ)));
          pr.TS0 = (uint32_t)std::max<uint64_t>(rb.TS0, pT * (uint32_t)(pt + (uint32_t)(rb.TS0 / pT)));
          pr.X1 = (uint32_t)std::min<uint64_t>(rb.X1, pX * (uint32_t)(px + (uint32_t)(rb.X0 / pX) + 1));
          pr.Y1 = (uint32_t)std::min<uint64_t>(rb.Y1, pY * (uint32_t)(py + (uint32_t)(rb.Y0 / pY) + 1));
          pr.Z1 = (uint32_t)std::min<uint64_t>(rb.Z1, pZ * (uint32_t)(pz + (uint32_t)(rb.Z0 / pZ) + 1));
          pr.TS1 = (uint32_t)std::min<uint64_t>(rb.TS1, pT * (uint32_t)(pt + (uint32_t)(rb.TS0 / pT) + 1));
          if ((c.nDecomp - c.decompX) < (int)r) {
            pr.X0 = prec_halve(pr.X0, (hb & kDimX) ? 1 : 0);
            pr.X1 = prec_halve(pr.X1, (hb & kDimX) ? 1 : 0);
          }
          if ((c.nDecomp - c.decompY) < (int)r) {
            pr.Y0 = prec_halve(pr.Y0, (hb & kDimY) ? 1 : 0);
            pr.Y1 = prec_halve(pr.Y1, (hb & kDimY) ? 1 : 0);
          }
          if ((c.nDecomp - c.decompZ) < (int)r) {
            pr.Z0 = prec_halve(pr.Z0, (hb & kDimZ) ? 1 : 0);
            pr.Z1 = prec_halve(pr.Z1, (hb & kDimZ) ? 1 : 0);
          }
          if ((c.nDecomp - c.decompTS) < (int)r) {
            pr.TS0 = prec_halve(pr.TS0, (hb & kDimTS) ? 1 : 0);
            pr.TS1 = prec_halve(pr.TS1, (hb & kDimTS) ? 1 : 0);
          }
          const Subband &s = par.subbands[sb_index];
          const uint32_t prec_index = (uint32_t)par.precincts.size();
          par.precincts.push_back(std::move(pr));
          Precinct &pp = par.precincts.back();
          if (init_precinct(c, par, pp, (uint32_t)((uint32_t)sbsX - s.box.X0),
                            (uint32_t)((uint32_t)sbsY - s.box.Y0),
                            (uint32_t)((uint32_t)sbsZ - s.box.Z0),
                            (uint32_t)((uint32_t)sbsT - s.box.TS0), sb_index, prec_index))
            return 1;
        }
  return 0;
}

uchar build_geometry(bwc_codec *codec) {
  const bwc_gl_ctrl &c = codec->control;
  const bwc_gl_inf &info = codec->info;
  // A geometry no device could hold (from a corrupt header, say) is refused before it is
  // built: building it codeblock by codeblock would run for hours, or exhaust host memory
  // (about 2 KB a codeblock).  The bound, 2^21 codeblocks at the field's codeblock size, is
  // over ten times the codeblocks of the largest field whose compression fits a B200's memory
  // (about 77 bytes of device memory a value, 32 x 32 x 16 codeblocks); likewise more than
  // 65536 tiles.
  {
    const uint64_t n[4] = {info.nX, info.nY, info.nZ, info.nTS};
    const uint64_t tsz[4] = {c.tileSizeX, c.tileSizeY, c.tileSizeZ, c.tileSizeTS};
    const uint8_t cb[4] = {c.cbX, c.cbY, c.cbZ, c.cbTS};
    double cells = info.nPar;
    bool empty = info.nPar == 0;
    for (int a = 0; a < 4; ++a) {
      empty = empty || n[a] == 0 || tsz[a] == 0;
      cells *= std::ceil((double)n[a] / std::ldexp(1.0, cb[a] < 63 ? cb[a] : 63));
    }
    if (empty || cells > (double)(1ull << 21) || c.nTiles > (1u << 16)) {
      warn(kMemError);
      return 1;
    }
  }
  free_engine(codec);
  bwc_b200_engine *eng = new (std::nothrow) bwc_b200_engine();
  if (!eng) {
    warn(kMemError);
    return 1;
  }
  codec->tile = eng;
  const uint32_t ntx = (uint32_t)std::ceil((double)((float)info.nX / (float)c.tileSizeX));
  const uint32_t nty = (uint32_t)std::ceil((double)((float)info.nY / (float)c.tileSizeY));
  const uint32_t ntz = (uint32_t)std::ceil((double)((float)info.nZ / (float)c.tileSizeZ));
  const uint32_t ntt = (uint32_t)std::ceil((double)((float)info.nTS / (float)c.tileSizeTS));
  eng->tiles.resize(c.nTiles);
  uint32_t i = 0;
  for (uint32_t t = 0; t < ntt; ++t)
    for (uint32_t z = 0; z < ntz; ++z)
      for (uint32_t y = 0; y < nty; ++y)
        for (uint32_t x = 0; x < ntx; ++x, ++i) {
          if (i >= eng->tiles.size()) return 1;
          Tile &tile = eng->tiles[i];
          uint64_t nPackets = 0;
          uint32_t max_Prec = 0;
          tile.index = i;
          tile.box.X0 = x * c.tileSizeX;
          tile.box.Y0 = y * c.tileSizeY;
          tile.box.Z0 = z * c.tileSizeZ;
          tile.box.TS0 = t * c.tileSizeTS;
          tile.box.X1 = std::min<uint64_t>(info.nX, (x + 1) * c.tileSizeX);
          tile.box.Y1 = std::min<uint64_t>(info.nY, (y + 1) * c.tileSizeY);
          tile.box.Z1 = std::min<uint64_t>(info.nZ, (z + 1) * c.tileSizeZ);
          tile.box.TS1 = std::min<uint64_t>(info.nTS, (t + 1) * c.tileSizeTS);
          tile.header_size = 18;
          tile.slope_max = 0x0000;
          tile.slope_min = 0xFFFF;
          tile.params.resize(info.nPar);
          for (uint8_t j = 0; j < info.nPar; ++j) {
            Parameter &par = tile.params[j];
            par.pmax = -kFltMax;
            par.pmin = kFltMax;
            par.box = tile.box;
            par.res.resize(c.nDecomp + 1);
            {
              // room for about the codeblocks the tile will have (codeblocks are large: growing
              // the vector a doubling at a time would move them several times)
              double cells = 1.0;
              const uint64_t ext[4] = {tile.box.nx(), tile.box.ny(), tile.box.nz(), tile.box.nt()};
              const uint8_t cbe[4] = {c.cbX, c.cbY, c.cbZ, c.cbTS};
              for (int a = 0; a < 4; ++a) cells *= std::ceil((double)ext[a] / std::ldexp(1.0, cbe[a]));
              par.codeblocks.reserve((size_t)(cells * 1.25) + 64);
            }
            for (int r = 0; r < c.nDecomp + 1; ++r) {
              Resolution &res = par.res[r];
              res.box.X0 = res_bound(par.box.X0, std::min<int>(c.nDecomp - r, c.decompX));
              res.box.Y0 = res_bound(par.box.Y0, std::min<int>(c.nDecomp - r, c.decompY));
              res.box.Z0 = res_bound(par.box.Z0, std::min<int>(c.nDecomp - r, c.decompZ));
              res.box.TS0 = res_bound(par.box.TS0, std::min<int>(c.nDecomp - r, c.decompTS));
              res.box.X1 = res_bound(par.box.X1, std::min<int>(c.nDecomp - r, c.decompX));
              res.box.Y1 = res_bound(par.box.Y1, std::min<int>(c.nDecomp - r, c.decompY));
              res.box.Z1 = res_bound(par.box.Z1, std::min<int>(c.nDecomp - r, c.decompZ));
              res.box.TS1 = res_bound(par.box.TS1, std::min<int>(c.nDecomp - r, c.decompTS));
              res.numPX = count_cells(res.box.X0, res.box.X1, 1ull << c.precSizeX);
              res.numPY = count_cells(res.box.Y0, res.box.Y1, 1ull << c.precSizeY);
              res.numPZ = count_cells(res.box.Z0, res.box.Z1, 1ull << c.precSizeZ);
              res.numPTS = count_cells(res.box.TS0, res.box.TS1, 1ull << c.precSizeTS);
              res.nprec = (uint64_t)res.numPX * res.numPY * res.numPZ * res.numPTS;
              nPackets += res.nprec * c.nLayers;
              max_Prec = (uint32_t)std::max<uint64_t>(res.nprec * c.nLayers, max_Prec);
              if (r == 0) {
                res.rcbX = std::min(c.cbX, (uint8_t)(c.precSizeX));
                res.rcbY = std::min(c.cbY, (uint8_t)(c.precSizeY));
                res.rcbZ = std::min(c.cbZ, (uint8_t)(c.precSizeZ));
                res.rcbTS = std::min(c.cbTS, (uint8_t)(c.precSizeTS));
              } else {
                res.rcbX = std::min(c.cbX, (uint8_t)(c.precSizeX - 1));
                res.rcbY = std::min(c.cbY, (uint8_t)(c.precSizeY - 1));
                res.rcbZ = std::min(c.cbZ, (uint8_t)(c.precSizeZ - 1));
                res.rcbTS = std::min(c.cbTS, (uint8_t)(c.precSizeTS - 1));
              }
              uint8_t hb = 0;
              hb |= (c.nDecomp - c.decompX < r && r > 0) ? kDimX : 0;
              hb |= (c.nDecomp - c.decompY < r && r > 0) ? kDimY : 0;
              hb |= (c.nDecomp - c.decompZ < r && r > 0) ? kDimZ : 0;
              hb |= (c.nDecomp - c.decompTS < r && r > 0) ? kDimTS : 0;
              int nsb = 1 << (((hb & kDimX)) + ((hb & kDimY) >> 1) + ((hb & kDimZ) >> 2) +
                              ((hb & kDimTS) >> 3));
              nsb -= (nsb & 1) ? 0 : 1;
              res.nsub = (uint8_t)nsb;
              res.first_subband = (uint32_t)par.subbands.size();
              res.packets.resize(res.nprec * c.nLayers);
              for (int l = 0, m = 0; m < nsb; ++l) {
                if (r == 0 || (((l & hb) == l) && l != 0)) {
                  const size_t cb_before = par.codeblocks.size();
                  if (init_subband(codec, par, r, (uint8_t)l)) return 1;
                  // packet descriptors for every codeblock added (libbwc.c:1663-1682)
                  for (size_t q = cb_before; q < par.codeblocks.size(); ++q) {
                    const Codeblock &cb = par.codeblocks[q];
                    const uint32_t p = cb.precinct - par.subbands.back().first_precinct;
                    for (int n = 0; n < c.nLayers; ++n) {
                      Packet &pk = res.packets[n * res.nprec + p];
                      pk.c = j;
                      pk.r = (uint8_t)r;
                      pk.p = p;
                      pk.l = (uint8_t)n;
                    }
                  }
                  m++;
                }
              }
            }
            for (Codeblock &cb : par.codeblocks) {
              cb.cp_mem.assign(c.nLayers + 1, 0);
              cb.beta = cb.beta_est = 3;
            }
          }
          tile.header_size += c.error_resilience ? (uint32_t)(8 * nPackets) : 0;
          tile.nPackets = nPackets;
          tile.max_Prec = max_Prec;
          tile.sequence.assign(nPackets, nullptr);
        }
  return 0;
}

}  // namespace bwcb

extern "C" uchar create_codec(bwc_codec *const codec) { return bwcb::build_geometry(codec); }

// ---------------------------------------------------------------------------------------------
// bwc_create_compression: rate string parsing (libbwc.c:2970-3131)
// ---------------------------------------------------------------------------------------------
static uchar bwc_create_compression_body(bwc_codec *const codec, bwc_stream *const stream, char *const rate_control);

extern "C" uchar bwc_create_compression(bwc_codec *const codec, bwc_stream *const stream,
                                        char *const rate_control) {
  return guarded<uchar>(1, [&] { return bwc_create_compression_body(codec, stream, rate_control); });
}

static uchar bwc_create_compression_body(bwc_codec *const codec, bwc_stream *const stream, char *const rate_control) {
  bwc_gl_ctrl *c = &codec->control;
  bwc_gl_inf *info = &codec->info;
  size_t size = 10;
  free(c->bitrate);
  c->bitrate = (float *)calloc(size, sizeof(float));
  if (!c->bitrate) {
    warn(kMemError);
    return 1;
  }
  char *save = nullptr;
  char *token = rate_control ? strtok_r(rate_control, "-, ", &save) : nullptr;
  if (!token) {
    c->bitrate[0] = kPrecBit + 1;
    c->nLayers = 1;
  } else {
    for (c->nLayers = 0; token; token = strtok_r(nullptr, "-, ", &save)) {
      float v = strtof(token, nullptr);
      if (v <= 0 || v > 64) {
        fprintf(stderr,
                "o##########################################################o\n"
                "|   ERROR: Invalid bitrate value: %-25f|\n"
                "|                                                          |\n"
                "|          The specified bitrate is not within its valid   |\n"
                "|          range of:                                       |\n"
                "|                                                          |\n"
                "|                        0 < Bitrate ≤ 64                  |\n"
                "|                                                          |\n"
                "o##########################################################o\n",
                v);
        return 1;
      }
      if (((int8_t)size - c->nLayers) == 0) {
        size += 10;
        c->bitrate = (float *)realloc(c->bitrate, size * sizeof(float));
      }
      // sorted insertion; values within 0.01 of an existing rate are dropped
      for (int8_t l = (int8_t)c->nLayers; l >= 0; --l) {
        if (l && v < c->bitrate[l - 1]) {
          c->bitrate[l] = c->bitrate[l - 1];
        } else if (l && std::fabs(v - c->bitrate[l - 1]) < 0.01f) {
          for (; l < c->nLayers; ++l) c->bitrate[l] = c->bitrate[l + 1];
          break;
        } else {
          c->bitrate[l] = v;
          c->nLayers++;
          break;
        }
      }
    }
  }
  c->bitrate = (float *)realloc(c->bitrate, c->nLayers * sizeof(float));
  // more than one tile: the geometry, rate control and codestream layout are built (and tested
  // against the reference through bwc_b200_assemble_tiles_from_tier1); bwc_compress and
  // bwc_b200_compress_batch refuse such codecs, the device path codes a single tile
  if (unsupported_kernel(*c, *info)) {
    warn("o##########################################################o\n"
         "| ERROR: this library implements the CDF 9/7 and LeGall    |\n"
         "|        5/3 wavelets only                                 |\n"
         "o##########################################################o\n");
    return 1;
  }
  if (c->quantization_style != bwc_qt_derived) {
    warn("o##########################################################o\n"
         "| ERROR: this library implements derived quantisation only |\n"
         "o##########################################################o\n");
    return 1;
  }
  if (create_codec(codec)) return 1;
  c->headerSize = 111 + (uint64_t)info->nPar * c->nTiles * 2 * kPrecByte + c->nLayers * 4;
  if (stream->codestream.aux) c->headerSize += 6 + stream->codestream.aux->size;
  if (stream->codestream.com) c->headerSize += 6 + stream->codestream.com->size;
  if (c->headerSize >= 0xFFFFFFFF) {
    warn("o==========================================================o\n"
         "| ERROR: Main header exceeds maximum size limit            |\n"
         "|                                                          |\n"
         "|        Appending the auxiliary information to the main   |\n"
         "|        header would exceed its maximum size limit of     |\n"
         "|        4294967295 bytes.                                 |\n"
         "|                                                          |\n"
         "o==========================================================o\n");
    return 1;
  }
  return 0;
}
