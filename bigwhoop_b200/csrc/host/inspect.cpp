// Host-only inspection entry points (declared in bwc_b200.h).
//
// They expose the codec geometry, the parsed state of a decompression codec, and the tier-2 +
// codestream stage on caller-supplied tier-1 results.  None of them codes samples: the
// compression and decompression paths proper run on the GPU only.
#include <cstring>

#include "bwc_b200.h"
#include "common.hpp"

using namespace bwcb;

static Parameter *param_of(bwc_codec *codec, uint8 p) {
  if (!codec || !codec->tile || codec->tile->tiles.empty()) return nullptr;
  Tile &t = codec->tile->tiles[0];
  return p < t.params.size() ? &t.params[p] : nullptr;
}

extern "C" int bwc_b200_codeblock_geometry(bwc_codec *const codec, uint8 const param,
                                           uint64 const c, uint64 *geom10) {
  Parameter *par = param_of(codec, param);
  if (!par || c >= par->codeblocks.size()) return 1;
  const Codeblock &cb = par->codeblocks[c];
  const Subband &sb = par->subbands[cb.subband];
  const uint64 g[10] = {cb.box.X0, cb.box.Y0, cb.box.Z0, cb.box.TS0, cb.box.X1,
                        cb.box.Y1, cb.box.Z1, cb.box.TS1, sb.highband, sb.Kmax};
  std::memcpy(geom10, g, sizeof(g));
  return 0;
}

extern "C" int bwc_b200_subband_steps(bwc_codec *const codec, uint8 const param, uint64 const c,
                                      double *out3) {
  Parameter *par = param_of(codec, param);
  if (!par || c >= par->codeblocks.size()) return 1;
  const Subband &sb = par->subbands[par->codeblocks[c].subband];
  out3[0] = sb.qt_eff;
  out3[1] = sb.qt_step;
  out3[2] = sb.dwt_gain;
  return 0;
}

extern "C" int bwc_b200_parsed_codeblock_of_tile(bwc_codec *const codec, uint32 const tile,
                                                 uint8 const param, uint64 const c,
                                                 int64 *meta3, uint64 *L) {
  if (!codec || !codec->tile || tile >= codec->tile->tiles.size()) return 1;
  Tile &t = codec->tile->tiles[tile];
  if (param >= t.params.size() || c >= t.params[param].codeblocks.size()) return 1;
  const Parameter &par = t.params[param];
  const Codeblock &cb = par.codeblocks[c];
  meta3[0] = par.subbands[cb.subband].Kmax - cb.enc.Kmsbs;
  meta3[1] = cb.enc.Kmsbs;
  meta3[2] = cb.enc.Z;
  if (L)
    for (int j = 0; j < kMaxPasses; ++j) L[j] = cb.enc.L[j];
  return 0;
}

extern "C" int bwc_b200_parsed_codeblock(bwc_codec *const codec, uint8 const param,
                                         uint64 const c, int64 *meta3, uint64 *L) {
  Parameter *par = param_of(codec, param);
  if (!par || c >= par->codeblocks.size()) return 1;
  const Codeblock &cb = par->codeblocks[c];
  meta3[0] = par->subbands[cb.subband].Kmax - cb.enc.Kmsbs;
  meta3[1] = cb.enc.Kmsbs;
  meta3[2] = cb.enc.Z;
  if (L)
    for (int j = 0; j < kMaxPasses; ++j) L[j] = cb.enc.L[j];
  return 0;
}

static size_t bwc_b200_assemble_from_tier1_body(bwc_codec *const codec, bwc_stream *const stream, uint8 const *K, uint8 const *Z, uint64 const *L, uint16 const *S, uint8 const *bytes, uint64 const *byte_offsets, bwc_float const *minmax, uint16 const slope_min, uint16 const slope_max);

extern "C" size_t bwc_b200_assemble_from_tier1(bwc_codec *const codec, bwc_stream *const stream,
                                               uint8 const *K, uint8 const *Z, uint64 const *L,
                                               uint16 const *S, uint8 const *bytes,
                                               uint64 const *byte_offsets,
                                               bwc_float const *minmax, uint16 const slope_min,
                                               uint16 const slope_max) {
  return guarded<size_t>(0, [&] { return bwc_b200_assemble_from_tier1_body(codec, stream, K, Z, L, S, bytes, byte_offsets, minmax, slope_min, slope_max); });
}

static size_t bwc_b200_assemble_from_tier1_body(bwc_codec *const codec, bwc_stream *const stream, uint8 const *K, uint8 const *Z, uint64 const *L, uint16 const *S, uint8 const *bytes, uint64 const *byte_offsets, bwc_float const *minmax, uint16 const slope_min, uint16 const slope_max) {
  if (!codec || !codec->tile || codec->tile->tiles.empty()) return 0;
  Tile &tile = codec->tile->tiles[0];
  uint64_t g = 0;
  for (size_t p = 0; p < tile.params.size(); ++p) {
    Parameter &par = tile.params[p];
    par.pmin = minmax[2 * p];
    par.pmax = minmax[2 * p + 1];
    for (Codeblock &cb : par.codeblocks) {
      CodedBlock &e = cb.enc;
      e.K = K[g];
      e.Z = Z[g];
      e.Kmsbs = e.K ? (uint8_t)(par.subbands[cb.subband].Kmax - e.K) : 0;
      for (int j = 0; j < e.Z; ++j) e.L[j] = (uint32_t)L[g * kMaxPasses + j];
      for (int j = 0; j <= e.Z; ++j) e.S[j] = S[g * (kMaxPasses + 1) + j];
      cb.data_off = byte_offsets[g];
      ++g;
    }
  }
  tile.slope_min = slope_min;
  tile.slope_max = slope_max;
  if (t2_encode(codec, tile)) return 0;
  std::vector<uint8_t> blob;
  std::vector<GatherPiece> pieces;
  const uint64_t total = layout_codestream(codec, stream, blob, pieces);
  if (!total) return 0;
  uint8_t *out = (uint8_t *)stream->out;
  for (const GatherPiece &pc : pieces)
    std::memcpy(out + pc.dst, (pc.from_blob ? blob.data() : bytes) + pc.src, pc.size);
  return total;
}

static size_t assemble_tiles_body(bwc_codec *const codec, bwc_stream *const stream,
                                  uint8 const *K, uint8 const *Z, uint64 const *L,
                                  uint16 const *S, uint8 const *bytes,
                                  uint64 const *byte_offsets, bwc_float const *minmax,
                                  uint16 const *slopes) {
  if (!codec || !codec->tile || codec->tile->tiles.empty()) return 0;
  uint64_t g = 0, tp = 0, t = 0;
  for (Tile &tile : codec->tile->tiles) {
    for (size_t p = 0; p < tile.params.size(); ++p, ++tp) {
      Parameter &par = tile.params[p];
      par.pmin = minmax[2 * tp];
      par.pmax = minmax[2 * tp + 1];
      for (Codeblock &cb : par.codeblocks) {
        CodedBlock &e = cb.enc;
        e.K = K[g];
        e.Z = Z[g];
        e.Kmsbs = e.K ? (uint8_t)(par.subbands[cb.subband].Kmax - e.K) : 0;
        for (int j = 0; j < e.Z; ++j) e.L[j] = (uint32_t)L[g * kMaxPasses + j];
        for (int j = 0; j <= e.Z; ++j) e.S[j] = S[g * (kMaxPasses + 1) + j];
        cb.data_off = byte_offsets[g];
        ++g;
      }
    }
    tile.slope_min = slopes[2 * t];
    tile.slope_max = slopes[2 * t + 1];
    ++t;
  }
  for (Tile &tile : codec->tile->tiles)
    if (t2_encode(codec, tile)) return 0;
  std::vector<uint8_t> blob;
  std::vector<GatherPiece> pieces;
  const uint64_t total = layout_codestream(codec, stream, blob, pieces);
  if (!total) return 0;
  uint8_t *out = (uint8_t *)stream->out;
  for (const GatherPiece &pc : pieces)
    std::memcpy(out + pc.dst, (pc.from_blob ? blob.data() : bytes) + pc.src, pc.size);
  return total;
}

extern "C" size_t bwc_b200_assemble_tiles_from_tier1(bwc_codec *const codec,
                                                     bwc_stream *const stream, uint8 const *K,
                                                     uint8 const *Z, uint64 const *L,
                                                     uint16 const *S, uint8 const *bytes,
                                                     uint64 const *byte_offsets,
                                                     bwc_float const *minmax,
                                                     uint16 const *slopes) {
  return guarded<size_t>(0, [&] {
    return assemble_tiles_body(codec, stream, K, Z, L, S, bytes, byte_offsets, minmax, slopes);
  });
}

extern "C" int bwc_b200_rate_features(bwc_codec *const codec, uint8 const layer, float *out) {
  if (!codec || !codec->tile || codec->tile->tiles.empty() || !out) return 1;
  const Tile &tile = codec->tile->tiles[0];
  if ((size_t)(layer + 1) * kRateFeatures > tile.rc_features.size()) return 1;
  std::memcpy(out, tile.rc_features.data() + (size_t)layer * kRateFeatures,
              kRateFeatures * sizeof(float));
  return 0;
}

extern "C" int bwc_b200_rate_stats(bwc_codec *const codec, uint8 const layer, double *out) {
  if (!codec || !codec->tile || codec->tile->tiles.empty() || !out) return 1;
  const Tile &tile = codec->tile->tiles[0];
  if ((size_t)(layer + 1) * kRateStats > tile.rc_stats.size()) return 1;
  std::memcpy(out, tile.rc_stats.data() + (size_t)layer * kRateStats, kRateStats * sizeof(double));
  return 0;
}
