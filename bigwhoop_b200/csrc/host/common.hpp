// Internal data model of the B200 BigWhoop codec (host side).
//
// The reference keeps its codec as a malloc'd pointer tree
// tile -> parameter -> resolution -> subband -> precinct -> codeblock
// (include/library/private/types.h:178-521).  Here the same geometry is stored as flat,
// index-linked tables per parameter, which is what the device kernels consume: one
// contiguous codeblock table in the reference's tier-1 order (libbwc.c:1639-1686), with
// subband and precinct tables referenced by index.
#pragma once

#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "bwc.h"

namespace bwcb {

#ifdef BWC_SINGLE_PRECISION
constexpr int     kPrecBit      = 31;
constexpr int     kPrecMantissa = 23;
constexpr int     kPrecByte     = 4;
constexpr bwc_raw kSignMask     = 0x80000000u;
constexpr bwc_raw kMantissaMask = 0x007FFFFFu;
constexpr bwc_raw kExponentMask = 0x7F800000u;
// prim_types_single.h:96 (the reference's own "FLT_MAX" for the single build)
constexpr bwc_float kFltMax = (bwc_float)1.70141183e+38;
#else
constexpr int     kPrecBit      = 63;
constexpr int     kPrecMantissa = 52;
constexpr int     kPrecByte     = 8;
constexpr bwc_raw kSignMask     = 0x8000000000000000ull;
constexpr bwc_raw kMantissaMask = 0x000FFFFFFFFFFFFFull;
constexpr bwc_raw kExponentMask = 0x7FF0000000000000ull;
constexpr bwc_float kFltMax = 1.7976931348623157e+308;
#endif
constexpr int kMaxPasses = MAXIMUM_NO_PASSES;
constexpr int kRateFeatures = 34;   // inputs of the rate-control warm start (tier2.cpp)
constexpr int kRateStats = 6;

// dimension flags of a subband's high-pass axes (macros.h:66-70)
constexpr uint8_t kDimX = 1, kDimY = 2, kDimZ = 4, kDimTS = 8;

// codestream markers (macros.h:73-88)
constexpr uint16_t kSOC = 0xFF50, kSGI = 0xFF51, kSGC = 0xFF52, kSAX = 0xFF53, kCOM = 0xFF57,
                   kEOH = 0xFF58, kSOT = 0xFF90, kSOP = 0xFF91, kEPH = 0xFF92, kSOD = 0xFF93,
                   kEOC = 0xFFFF;

struct Box {
  uint64_t X0 = 0, Y0 = 0, Z0 = 0, TS0 = 0;
  uint64_t X1 = 0, Y1 = 0, Z1 = 0, TS1 = 0;
  uint64_t nx() const { return X1 - X0; }
  uint64_t ny() const { return Y1 - Y0; }
  uint64_t nz() const { return Z1 - Z0; }
  uint64_t nt() const { return TS1 - TS0; }
  uint64_t size() const { return nx() * ny() * nz() * nt(); }
};

// 4D quad tree over the codeblocks of one precinct (tagtree.c:196-298).  Nodes are stored
// level by level, leaves first; `parent` indexes into `nodes` (-1 at the root).
struct TagNode {
  uint16_t value = 0xFFFF;
  uint16_t threshold = 0;
  int64_t parent = -1;
};

struct TagTree {
  uint64_t leaves = 0;
  std::vector<TagNode> nodes;
};

// Per-codeblock tier-1 result as tier-2 sees it (types.h:178-189).
struct CodedBlock {
  uint8_t K = 0;
  uint8_t Kmsbs = 0;
  uint8_t Z = 0;
  uint32_t L[kMaxPasses] = {};   // cumulative codeword bytes after each pass (< 4 GiB)
  uint16_t S[kMaxPasses + 1] = {};
};

struct Codeblock {
  Box box;                 // position in the parameter's working buffer (Mallat layout)
  uint32_t subband = 0;    // index into Parameter::subbands
  uint32_t precinct = 0;   // index into Parameter::precincts
  uint32_t idx = 0;        // index inside its precinct (tag-tree leaf)
  // tier-2 control (types.h:203-212)
  uint16_t beta = 3, beta_est = 3;
  std::vector<int16_t> cp_mem;   // nLayers + 1 entries, cp_mem[0] == 0 always
  int16_t *cp() { return cp_mem.data() + 1; }
  CodedBlock enc;
  // where the codeblock's coded bytes live
  uint64_t data_off = 0;   // compress: byte offset in the device tier-1 buffer
  uint64_t data_cap = 0;   // compress: capacity of that region
  // decompress: chunks of the codeblock's bytes inside the codestream (offset, size)
  std::vector<std::pair<uint64_t, uint32_t>> chunks;
};

struct Precinct {
  uint32_t X0 = 0, Y0 = 0, Z0 = 0, TS0 = 0, X1 = 0, Y1 = 0, Z1 = 0, TS1 = 0;
  uint16_t numCbX = 0, numCbY = 0, numCbZ = 0, numCbTS = 0;
  uint64_t ncb = 0;
  uint64_t first_cb = 0;   // index into Parameter::codeblocks
  TagTree incl, msbs;
};

struct Subband {
  Box box;
  bwc_float dwt_gain = 0;
  uint8_t highband = 0;
  uint16_t Kmax = 0;
  uint16_t qt_mantissa = 0;
  uint8_t qt_exponent = 0;
  bwc_float qt_eff = 0;     // qt_effective_step_size
  bwc_float qt_step = 0;    // qt_step_size
  uint32_t first_precinct = 0;   // precincts of this subband: [first, first + res.nprec)
};

struct Packet {
  std::vector<uint8_t> header;
  uint64_t body_size = 0;
  uint8_t e = 0;
  uint64_t size = 0;
  uint32_t p = 0;
  uint8_t c = 0, l = 0, r = 0;
  // compression: the body as (byte offset in the device tier-1 buffer, size) pieces
  std::vector<std::pair<uint64_t, uint32_t>> pieces;
  // parsing: where the packet's body starts in the input codestream
  uint64_t body_pos = 0;
  uint64_t header_pos = 0;
  uint64_t header_len = 0;
};

struct Resolution {
  Box box;
  uint16_t numPX = 0, numPY = 0, numPZ = 0, numPTS = 0;
  uint64_t nprec = 0;
  uint8_t rcbX = 0, rcbY = 0, rcbZ = 0, rcbTS = 0;
  uint8_t nsub = 0;
  uint32_t first_subband = 0;
  std::vector<Packet> packets;   // nprec * nLayers, index l * nprec + p
};

struct Parameter {
  Box box;
  bwc_float pmin = 0, pmax = 0;
  bwc_float alpha = 0, beta = 0;
  std::vector<Resolution> res;
  std::vector<Subband> subbands;
  std::vector<Precinct> precincts;
  std::vector<Codeblock> codeblocks;   // tier-1 order
};

struct Tile {
  Box box;
  uint32_t index = 0;
  uint64_t body_size = 0;
  uint32_t header_size = 0;
  uint64_t nPackets = 0;
  uint32_t max_Prec = 0;
  uint16_t slope_min = 0xFFFF, slope_max = 0;
  std::vector<Parameter> params;
  std::vector<Packet *> sequence;
  // rate control of the last compression, per quality layer
  std::vector<float> rc_features;   // kRateFeatures per layer (the warm start's inputs)
  std::vector<double> rc_stats;     // kRateStats per layer, see tier2.cpp
};

struct DeviceState;   // CUDA resources (api.cpp)

}  // namespace bwcb

struct bwc_b200_engine {
  std::vector<bwcb::Tile> tiles;
  bwcb::DeviceState *dev = nullptr;
};

namespace bwcb {

// ---- setup (codec.cpp) ------------------------------------------------------------------
uchar initialize_gain_lut();
bwc_float dwt_energy_gain(const bwc_gl_ctrl &control, uchar highband, uint16_t level);
void reset_gain_lut();
void copy_gain_lut(double *out30);
uchar build_geometry(bwc_codec *codec);   // create_codec
void free_engine(bwc_codec *codec);

// ---- bit I/O and tag trees (bitio.cpp) ------------------------------------------------------
struct RawBits;

struct BitWriter {
  std::vector<uint8_t> mem;
  uint8_t T = 0;
  int8_t t = 8;
  uint64_t L() const { return mem.size(); }
  // one bit, most significant first; a byte after 0xFF holds 7 bits (bit stuffing)
  void emit(uint64_t bit) {
    t--;
    if (bit) T |= (uint8_t)(1u << t);
    if (!t) {
      mem.push_back(T);
      t = (T == 0xFF) ? 7 : 8;
      T = 0;
    }
  }
  void flush();
  // every bit of an unstuffed bit string, as emit() would write them one by one
  void append(const RawBits &rb);
  uint64_t bytes_used() const { return T == 0xFF ? mem.size() + 1 : mem.size(); }
};

struct BitReader {
  const uint8_t *mem = nullptr;
  uint64_t L = 0, Lmax = 0;
  uint16_t T = 0;
  int8_t t = 0;
  uchar error = 0;
  uchar get_bit();
  uint64_t get_symbol(uint8_t nbytes);
  bool can_read(uint64_t n) const { return L + n <= Lmax; }
  uint64_t bytes_used() const { return T == 0xFF ? L + 1 : L; }
};

// Unstuffed bit string (most-significant bit first), for header pieces that are assembled
// and stuffed later.
struct RawBits {
  std::vector<uint64_t> words;
  uint64_t n = 0;
  void emit(uint64_t bit) {
    if ((n & 63) == 0) words.push_back(0);
    if (bit) words.back() |= 1ull << (63 - (n & 63));
    ++n;
  }
  void clear() {
    words.clear();
    n = 0;
  }
};

void tagtree_init(TagTree &tt, uint64_t lx, uint64_t ly, uint64_t lz, uint64_t lts);
void tagtree_reset(TagTree &tt);
void tagtree_set(TagTree &tt, uint64_t leaf, uint16_t value);
void tagtree_encode(TagTree &tt, BitWriter &bw, uint32_t threshold, uint64_t leaf, uchar estimate);
// the same bits, unstuffed (byte stuffing is applied when they are appended to a BitWriter)
void tagtree_encode_bits(TagTree &tt, RawBits &out, uint32_t threshold, uint64_t leaf,
                         uchar estimate);
// the bits an estimating tagtree_encode would emit (the tree is left unchanged)
void tagtree_estimate(const TagTree &tt, RawBits &out, uint32_t threshold, uint64_t leaf);
uchar tagtree_decode(TagTree &tt, BitReader &br, uint32_t threshold, uint64_t leaf);
bool tagtree_decode_until_known(TagTree &tt, BitReader &br, uint64_t leaf, uint32_t tmax);

// ---- tier 2 and codestream (tier2.cpp, codestream.cpp) ------------------------------------------
uchar t2_encode(bwc_codec *codec, Tile &tile);
extern thread_local bool t_rate_control_in_parallel_fields;
// fn(i) for every i in [0, n) on the host thread pool of tier 2 (and the calling thread)
void host_parallel(size_t n, const std::function<void(size_t)> &fn);
uchar parse_packet(bwc_codec *codec, Tile &tile, Packet &packet, const uint8_t *cs,
                   uint64_t cs_len, uint64_t pos, uint64_t body_size);
uchar sequence_packets(bwc_codec *codec, Tile &tile);
// writes header + packet headers into `blob`, records body pieces for the device gather
struct GatherPiece {
  uint64_t src;   // byte offset in the source (blob or device tier-1 buffer)
  uint64_t dst;   // byte offset in the codestream
  uint32_t size;
  uint32_t from_blob;   // 1: source is the host-built blob, 0: device tier-1 buffer
};
uint64_t layout_codestream(bwc_codec *codec, bwc_stream *data, std::vector<uint8_t> &blob,
                           std::vector<GatherPiece> &pieces);
uchar parse_main_header(bwc_codec *codec, bwc_stream *data, BitReader &br);
uchar parse_codestream(bwc_codec *codec, bwc_stream *data, uint8_t layer);

// ---- helpers ---------------------------------------------------------------------------------
void warn(const char *msg);
extern const char *kMemError;
extern const char *kCsError;

// No C++ exception may cross the C API (a corrupt codestream can ask for an impossible
// geometry, and std::bad_alloc would end the caller's process): every entry point that
// allocates runs its body through this and returns `on_error` instead, after the reference's
// memory-error message.
template <class R, class F>
R guarded(R on_error, F &&body) noexcept {
  try {
    return body();
  } catch (...) {
    warn(kMemError);
  }
  return on_error;
}

// true when an axis that the transform decomposes (levels > 0, more than one sample) uses a
// wavelet kernel this library does not implement: Haar (the reference has no boundary extension
// for it, dwt.c:1259-1262, so it cannot transform such a field) or a value outside the enum
bool unsupported_kernel(const bwc_gl_ctrl &c, const bwc_gl_inf &info);

}  // namespace bwcb
