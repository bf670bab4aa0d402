// Codestream layout and parsing.
//
// Main header: SOC, Lcss, SGI (dimensions and precisions), SGC (the setter bitmask CSsgc and
// every control value), optional SAX/COM, EOH and the per-parameter min/max as raw bwc_float
// bits (codestream.c:140-277).  Tile: SOT, 14, index, body size, SOD, then the packets in
// sequence order, each optionally wrapped in SOP/EPH (codestream.c:508-570).  All progression
// orders except RLCP are laid out as LRCP, as in the reference (codestream.c:344-470).
//
// Compression does not copy packet bodies on the host: the layout is emitted as a list of
// pieces, host-built header bytes plus (offset, size) slices of the device tier-1 buffer, which
// one device gather turns into the final codestream.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.hpp"

namespace bwcb {

namespace {
struct ByteSink {
  std::vector<uint8_t> &blob;
  std::vector<GatherPiece> &pieces;
  uint64_t pos = 0;
  void sym(uint64_t v, int n) {
    for (int i = n; i-- > 0;) byte((uint8_t)(v >> (8 * i)));
  }
  void byte(uint8_t b) {
    if (pieces.empty() || !pieces.back().from_blob ||
        pieces.back().src + pieces.back().size != blob.size() ||
        pieces.back().dst + pieces.back().size != pos) {
      pieces.push_back({blob.size(), pos, 0, 1});
    }
    blob.push_back(b);
    pieces.back().size++;
    pos++;
  }
  void chunk(const uint8_t *p, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) byte(p[i]);
  }
  void device(uint64_t src, uint32_t n) {
    if (!n) return;
    pieces.push_back({src, pos, n, 0});
    pos += n;
  }
};
}  // namespace

uchar sequence_packets(bwc_codec *codec, Tile &tile) {
  const bwc_gl_ctrl &c = codec->control;
  uint64_t size = 0, idx = 0;
  auto visit = [&](Parameter &par, int r, int l) {
    Resolution &res = par.res[r];
    for (uint64_t p = 0; p < res.nprec; ++p, ++idx) {
      Packet *pk = &res.packets[(uint64_t)l * res.nprec + p];
      if (idx < tile.sequence.size()) tile.sequence[idx] = pk;
      size += pk->size;
      if (c.error_resilience) size += 6;
    }
  };
  if (c.progression == bwc_prog_RLCP) {
    for (int r = 0; r < c.nDecomp + 1; ++r)
      for (int l = 0; l < c.nLayers; ++l)
        for (Parameter &par : tile.params) visit(par, r, l);
  } else if (c.progression <= bwc_prog_CPRL) {
    for (int l = 0; l < c.nLayers; ++l)
      for (int r = 0; r < c.nDecomp + 1; ++r)
        for (Parameter &par : tile.params) visit(par, r, l);
  } else {
    return 1;
  }
  tile.body_size = size;
  return 0;
}

static void write_main_header(bwc_codec *codec, bwc_stream *data, ByteSink &s) {
  bwc_gl_inf &info = codec->info;
  bwc_gl_ctrl &c = codec->control;
  bwc_span *aux = data->codestream.aux, *com = data->codestream.com;
  s.sym(kSOC, 2);
  s.sym(c.codestreamSize, 8);
  s.sym(kSGI, 2);
  s.sym(31, 2);
  s.sym(info.nX, 8);
  s.sym(info.nY, 8);
  s.sym(info.nZ, 8);
  s.sym(info.nTS, 8);
  s.sym(info.nPar, 1);
  s.sym((uint8_t)info.data_prec, 1);
  s.sym((uint8_t)info.codec_prec, 1);
  s.sym(kSGC, 2);
  s.sym(50 + c.nLayers * 4, 2);
  s.sym(c.CSsgc, 2);
  s.sym(c.error_resilience, 1);
  s.sym(c.quantization_style, 1);
  s.sym(c.guard_bits, 1);
  s.sym(c.qt_exponent, 1);
  s.sym(c.qt_mantissa, 2);
  s.sym(c.progression, 1);
  s.sym((c.KernelX << 6 | c.KernelY << 4 | c.KernelZ << 2 | c.KernelTS) & 0xFF, 1);
  s.sym(c.decompX, 1);
  s.sym(c.decompY, 1);
  s.sym(c.decompZ, 1);
  s.sym(c.decompTS, 1);
  s.sym((c.precSizeY << 4 | c.precSizeX) & 0xFF, 1);
  s.sym((c.precSizeTS << 4 | c.precSizeZ) & 0xFF, 1);
  s.sym(c.cbX, 1);
  s.sym(c.cbY, 1);
  s.sym(c.cbZ, 1);
  s.sym(c.cbTS, 1);
  s.sym(c.Qm, 1);
  s.sym(c.tileSizeX, 8);
  s.sym(c.tileSizeY, 8);
  s.sym(c.tileSizeZ, 8);
  s.sym(c.tileSizeTS, 8);
  s.sym(c.nLayers, 1);
  for (int l = 0; l < c.nLayers; ++l) {
    uint32_t bits;
    std::memcpy(&bits, &c.bitrate[l], 4);
    s.sym(bits, 4);
  }
  if (aux) {
    s.sym(kSAX, 2);
    s.sym((uint32_t)(aux->size + 4), 4);
    s.chunk(aux->memory, aux->size);
  }
  if (com) {
    s.sym(kCOM, 2);
    s.sym((uint16_t)(com->size + 2), 2);
    s.chunk(com->memory, com->size);
  }
  s.sym(kEOH, 2);
  s.sym((uint16_t)(info.nPar * c.nTiles * 2 * kPrecByte), 2);
  for (Tile &tile : codec->tile->tiles) {
    for (Parameter &par : tile.params) {
      bwc_raw mn, mx;
      std::memcpy(&mn, &par.pmin, sizeof(bwc_raw));
      std::memcpy(&mx, &par.pmax, sizeof(bwc_raw));
      s.sym(mn, kPrecByte);
      s.sym(mx, kPrecByte);
      par.pmax = -kFltMax;
      par.pmin = kFltMax;
    }
  }
}

uint64_t layout_codestream(bwc_codec *codec, bwc_stream *data, std::vector<uint8_t> &blob,
                           std::vector<GatherPiece> &pieces) {
  bwc_gl_ctrl &c = codec->control;
  blob.clear();
  pieces.clear();
  c.codestreamSize = c.headerSize + 2;
  for (Tile &tile : codec->tile->tiles) {
    if (sequence_packets(codec, tile)) return 0;
    c.codestreamSize += tile.header_size + tile.body_size;
  }
  ByteSink s{blob, pieces};
  write_main_header(codec, data, s);
  for (Tile &tile : codec->tile->tiles) {
    s.sym(kSOT, 2);
    s.sym(14, 2);
    s.sym(tile.index, 4);
    s.sym(tile.body_size, 8);
    s.sym(kSOD, 2);
    for (uint64_t i = 0; i < tile.nPackets; ++i) {
      Packet *pk = tile.sequence[i];
      if (c.error_resilience) {
        s.sym(kSOP, 2);
        s.sym(4, 2);
        s.sym(i % 0x100000000ull, 4);
      }
      if (!pk->header.empty()) {
        s.chunk(pk->header.data(), pk->header.size());
        if (c.error_resilience) s.sym(kEPH, 2);
        pk->header.clear();
      }
      for (auto &pc : pk->pieces) s.device(pc.first, pc.second);
      pk->pieces.clear();
      pk->body_size = 0;
    }
  }
  s.sym(kEOC, 2);
  if (s.pos > c.codestreamSize) {
    // the reference stops writing once its precomputed size is exhausted
    warn(kCsError);
    return 0;
  }
  return s.pos;
}

// ---------------------------------------------------------------------------------------------
// Parsing (codestream.c:601-1512)
// ---------------------------------------------------------------------------------------------
uchar parse_main_header(bwc_codec *codec, bwc_stream *data, BitReader &br) {
  bwc_gl_ctrl &c = codec->control;
  bwc_gl_inf &info = codec->info;
  bool sgi = false, sgc = false;
  bwc_precision codec_prec = bwc_precision_double;
  uint8_t index = 0;
  while (br.can_read(2)) {
    const uint16_t marker = (uint16_t)br.get_symbol(2);
    if (marker < 0xFF00) {
      warn(kCsError);
      return 1;
    }
    switch (marker) {
      case kSOC: {
        if (index != 0 && !br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        br.Lmax = br.get_symbol(8);
        break;
      }
      case kSGI: {
        if (index != 1 && !br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Linf = (uint16_t)br.get_symbol(2);
        if (!br.can_read((uint64_t)(uint16_t)(Linf - 2))) {
          warn(kCsError);
          return 1;
        }
        const uint64_t nX = br.get_symbol(8), nY = br.get_symbol(8), nZ = br.get_symbol(8),
                       nTS = br.get_symbol(8);
        const uint8_t nPar = (uint8_t)br.get_symbol(1);
        const bwc_precision dp = (bwc_precision)br.get_symbol(1);
        codec_prec = (bwc_precision)br.get_symbol(1);
        info.codec_prec = codec_prec;
        if (!configure_codec(codec, nX, nY, nZ, nTS, nPar, dp)) return 1;
        c.codestreamSize = br.Lmax;
        sgi = true;
        break;
      }
      case kSGC: {
        if (index != 2 && !br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Lctr = (uint16_t)br.get_symbol(2);
        if (!br.can_read((uint64_t)(uint16_t)(Lctr - 2))) {
          warn(kCsError);
          return 1;
        }
        const uint16_t CSsgc = (uint16_t)br.get_symbol(2);
        uint64_t v = br.get_symbol(1);
        if (CSsgc & (1 << 0)) bwc_set_error_resilience(codec);
        v = br.get_symbol(1);
        if (CSsgc & (1 << 1)) set_quant_style(codec, (bwc_quant_st)v);
        v = br.get_symbol(1);   // guard bits: stored, not restored (codestream.c:756)
        const uint32_t exponent = (uint32_t)br.get_symbol(1);
        const uint32_t mantissa = (uint32_t)br.get_symbol(2);
        if (CSsgc & (1 << 2)) {
          c.qt_exponent = exponent;
          c.qt_mantissa = mantissa;
        }
        v = br.get_symbol(1);
        if (CSsgc & (1 << 3)) set_progression(codec, (bwc_prog_ord)(uint8_t)v);
        v = br.get_symbol(1);
        if (CSsgc & (1 << 4))
          set_kernels(codec, (bwc_dwt_filter)(0x03 & (v >> 6)), (bwc_dwt_filter)(0x03 & (v >> 4)),
                      (bwc_dwt_filter)(0x03 & (v >> 2)), (bwc_dwt_filter)(0x03 & v));
        v = br.get_symbol(4);
        if (CSsgc & (1 << 5))
          bwc_set_decomp(codec, (uint8_t)(v >> 24), (uint8_t)(v >> 16), (uint8_t)(v >> 8),
                         (uint8_t)v);
        v = br.get_symbol(2);
        if (CSsgc & (1 << 6))
          bwc_set_precincts(codec, (uint8_t)(0x0F & (v >> 8)), (uint8_t)(0x0F & (v >> 12)),
                            (uint8_t)(0x0F & v), (uint8_t)(0x0F & (v >> 4)));
        v = br.get_symbol(4);
        if (CSsgc & (1 << 7))
          bwc_set_codeblocks(codec, (uint8_t)(v >> 24), (uint8_t)(v >> 16), (uint8_t)(v >> 8),
                             (uint8_t)v);
        v = br.get_symbol(1);
        if (CSsgc & (1 << 8)) bwc_set_qm(codec, (uint8_t)v);
        const uint64_t tX = br.get_symbol(8), tY = br.get_symbol(8), tZ = br.get_symbol(8),
                       tT = br.get_symbol(8);
        if (CSsgc & (1 << 9)) bwc_set_tiles(codec, tX, tY, tZ, tT, bwc_tile_sizeof);
        c.nLayers = (uint8_t)br.get_symbol(1);
        free(c.bitrate);
        c.bitrate = (float *)calloc(c.nLayers ? c.nLayers : 1, sizeof(float));
        if (!c.bitrate) {
          warn(kMemError);
          return 1;
        }
        for (int l = 0; l < c.nLayers; ++l) {
          const uint32_t bits = (uint32_t)br.get_symbol(4);
          std::memcpy(&c.bitrate[l], &bits, 4);
        }
        // more than one tile: parsed here (tested against the reference's parser);
        // bwc_decompress refuses such codecs, the device path decodes a single tile
        if (unsupported_kernel(c, info)) {
          warn("o##########################################################o\n"
               "| ERROR: this library implements the CDF 9/7 and LeGall    |\n"
               "|        5/3 wavelets only                                 |\n"
               "o##########################################################o\n");
          return 1;
        }
        if (c.quantization_style != bwc_qt_derived) {
          warn("o##########################################################o\n"
               "| ERROR: this library implements derived quantisation only |\n"
               "o##########################################################o\n");
          return 1;
        }
        if (build_geometry(codec)) return 1;
        sgc = true;
        break;
      }
      case kSAX: {
        if (index <= 2 && !br.can_read(4)) {
          warn(kCsError);
          return 1;
        }
        const uint32_t Lsax = (uint32_t)br.get_symbol(4);
        if (Lsax < 4 || !br.can_read(Lsax - 4)) {
          warn(kCsError);
          return 1;
        }
        if (bwc_set_aux(data, (const char *)br.mem + br.L, Lsax - 4)) return 1;
        br.L += Lsax - 4;
        break;
      }
      case kCOM: {
        if (index <= 2 && !br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Lcom = (uint16_t)br.get_symbol(2);
        if (Lcom < 2 || !br.can_read((uint64_t)(Lcom - 2))) {
          warn(kCsError);
          return 1;
        }
        if (bwc_set_com(data, (const char *)br.mem + br.L, (uint16_t)(Lcom - 2))) return 1;
        br.L += Lcom - 2;
        break;
      }
      case kEOH: {
        if (!(sgi && sgc)) {
          warn(kCsError);
          return 1;
        }
        if (index <= 2 && !br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Leoh = (uint16_t)br.get_symbol(2);
        if (!br.can_read((uint64_t)(uint16_t)(Leoh - 2))) {
          warn(kCsError);
          return 1;
        }
        for (Tile &tile : codec->tile->tiles) {
          for (Parameter &par : tile.params) {
            if (codec_prec == bwc_precision_double) {
              uint64_t a = br.get_symbol(8), b = br.get_symbol(8);
              double fa, fb;
              std::memcpy(&fa, &a, 8);
              std::memcpy(&fb, &b, 8);
              par.pmin = (bwc_float)fa;
              par.pmax = (bwc_float)fb;
            } else if (codec_prec == bwc_precision_single) {
              uint32_t a = (uint32_t)br.get_symbol(4), b = (uint32_t)br.get_symbol(4);
              float fa, fb;
              std::memcpy(&fa, &a, 4);
              std::memcpy(&fb, &b, 4);
              par.pmin = (bwc_float)fa;
              par.pmax = (bwc_float)fb;
            }
          }
        }
        return br.error ? 1 : 0;
      }
      default: {
        if (!br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Lunk = (uint16_t)br.get_symbol(2);
        if (Lunk < 2 || !br.can_read((uint64_t)(Lunk - 2))) {
          warn(kCsError);
          return 1;
        }
        br.L += Lunk - 2;
        break;
      }
    }
    if (br.error) {
      warn(kCsError);
      return 1;
    }
    index++;
  }
  return 1;
}

static uchar parse_tile(bwc_codec *codec, BitReader &br, const uint8_t *cs, uint64_t cs_len) {
  bwc_gl_ctrl &c = codec->control;
  if (!br.can_read(2)) {
    warn(kCsError);
    return 1;
  }
  const uint16_t L = (uint16_t)br.get_symbol(2);
  if (!br.can_read((uint64_t)(uint16_t)(L - 2))) {
    warn(kCsError);
    return 1;
  }
  const uint32_t t = (uint32_t)br.get_symbol(4);
  if (t >= c.nTiles) {
    warn(kCsError);
    return 1;
  }
  Tile &tile = codec->tile->tiles[t];
  uint64_t body_size = br.get_symbol(8);
  tile.body_size = body_size;
  if (kSOD != (uint16_t)br.get_symbol(2)) {
    warn(kCsError);
    return 1;
  }
  if (sequence_packets(codec, tile)) return 1;
  uint64_t idx = 0;
  while (body_size != 0 && br.can_read(body_size) && idx < tile.nPackets) {
    if (kSOP == (uint16_t)br.get_symbol(2)) {
      if (!br.can_read(6)) {
        warn(kCsError);
        return 1;
      }
      if (4 != (uint16_t)br.get_symbol(2)) {
        warn(kCsError);
        return 1;
      }
      br.get_symbol(4);
      body_size -= 8;
    } else {
      br.L -= 2;
    }
    Packet *pk = tile.sequence[idx++];
    if (parse_packet(codec, tile, *pk, cs, cs_len, br.L, body_size)) {
      warn(kCsError);
      return 1;
    }
    br.L += pk->size;
    body_size -= pk->size;
  }
  return 0;
}

uchar parse_codestream(bwc_codec *codec, bwc_stream *data, uint8_t layer) {
  BitReader br;
  br.mem = (const uint8_t *)data->inp;
  br.Lmax = 10;
  if (parse_main_header(codec, data, br)) return 1;
  codec->control.useLayer = codec->control.nLayers - 1;
  if (layer < codec->control.nLayers && layer > 0) codec->control.useLayer = layer;
  const uint64_t cs_len = br.Lmax;
  while (br.can_read(2)) {
    const uint16_t marker = (uint16_t)br.get_symbol(2);
    if (marker < 0xFF00) {
      warn(kCsError);
      return 1;
    }
    switch (marker) {
      case kSOT:
        if (parse_tile(codec, br, (const uint8_t *)data->inp, cs_len)) return 1;
        break;
      case kEOC:
        return 0;
      case kSOC: case kSGI: case kSGC: case kSAX: case kCOM: case kEOH:
        warn(kCsError);
        return 1;
      default: {
        if (!br.can_read(2)) {
          warn(kCsError);
          return 1;
        }
        const uint16_t Lunk = (uint16_t)br.get_symbol(2);
        if (Lunk < 2 || !br.can_read((uint64_t)(Lunk - 2))) {
          warn(kCsError);
          return 1;
        }
        br.L += Lunk - 2;
        break;
      }
    }
  }
  return 0;
}

}  // namespace bwcb

using namespace bwcb;

static bwc_header * bwc_open_header_body(void *const inpbuf);

extern "C" bwc_header *bwc_open_header(void *const inpbuf) {
  return guarded<bwc_header *>(nullptr, [&] { return bwc_open_header_body(inpbuf); });
}

static bwc_header * bwc_open_header_body(void *const inpbuf) {
  bwc_stream *data = bwc_init_stream(inpbuf, nullptr, decomp);
  bwc_codec *codec = bwc_alloc_decoder();
  if (!data || !codec) {
    free(data);
    bwc_free_codec(codec);
    return nullptr;
  }
  BitReader br;
  br.mem = (const uint8_t *)inpbuf;
  br.Lmax = 10;
  if (parse_main_header(codec, data, br)) {
    bwc_free_codec(codec);
    free(data);
    return nullptr;
  }
  bwc_header *h = (bwc_header *)calloc(1, sizeof(bwc_header));
  if (!h) {
    warn(kMemError);
    bwc_free_codec(codec);
    free(data);
    return nullptr;
  }
  h->info = codec->info;
  h->control = codec->control;
  h->control.bitrate = (float *)calloc(codec->control.nLayers ? codec->control.nLayers : 1, sizeof(float));
  if (!h->control.bitrate) {
    warn(kMemError);
    bwc_free_codec(codec);
    free(data);
    free(h);
    return nullptr;
  }
  std::memcpy(h->control.bitrate, codec->control.bitrate, codec->control.nLayers * sizeof(float));
  bwc_free_codec(codec);
  if (data->codestream.aux) {
    h->aux.memory = data->codestream.aux->memory;
    h->aux.size = data->codestream.aux->size;
    free(data->codestream.aux);
  }
  if (data->codestream.com) {
    h->com.memory = data->codestream.com->memory;
    h->com.size = data->codestream.com->size;
    free(data->codestream.com);
  }
  free(data);
  return h;
}

extern "C" void bwc_close_header(bwc_header *const header) {
  if (!header) return;
  free(header->aux.memory);
  free(header->com.memory);
  free(header->control.bitrate);
  free(header);
}

static uchar bwc_create_decompression_body(bwc_codec *const codec, bwc_stream *const stream, uint8 const layer);

extern "C" uchar bwc_create_decompression(bwc_codec *const codec, bwc_stream *const stream,
                                          uint8 const layer) {
  return guarded<uchar>(1, [&] { return bwc_create_decompression_body(codec, stream, layer); });
}

static uchar bwc_create_decompression_body(bwc_codec *const codec, bwc_stream *const stream, uint8 const layer) {
  if (!codec || !stream) return 1;
  return parse_codestream(codec, stream, layer) ? 1 : 0;
}
