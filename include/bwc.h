/*
 * bwc.h -- public C interface of the B200 implementation of the BigWhoop (libbwc) codec.
 *
 * Drop-in for the reference's generated public header (public_header.py concatenates
 * include/library/private/*.h into include/library/public/bwc.h).  Every function declared
 * below has the prototype of its reference counterpart (include/library/private/libbwc.h:67-161)
 * and the structs a caller reads directly -- bwc_span, bwc_gl_inf, bwc_stream, bwc_gl_ctrl,
 * bwc_header and bwc_codec -- have the reference's field order and types
 * (include/library/private/types.h:89-600), so code written against libbwc compiles and links
 * against this library unchanged.  The codec's internal tile tree is not exposed: bwc_codec's
 * `tile` member points to the library's own opaque state.
 *
 * Like the reference, the codec's floating-point type is fixed when the library is built:
 * define BWC_SINGLE_PRECISION for the single-precision library (bwc_float = float, 31
 * bit planes), otherwise bwc_float = double with 63 bit planes
 * (include/library/private/prim_types_{double,single}.h).
 *
 * Additional, non-reference entry points (device-resident buffers, batches, stage access)
 * are declared in bwc_b200.h.
 */
#ifndef BWC_H
#define BWC_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- primitive types (prim_types_*.h:58-78) ---------------------------------------------- */
typedef unsigned char  uchar;
typedef unsigned short ushort;
typedef unsigned int   uint;
typedef int8_t         int8;
typedef uint8_t        uint8;
typedef int16_t        int16;
typedef uint16_t       uint16;
typedef int32_t        int32;
typedef uint32_t       uint32;
typedef int64_t        int64;
typedef uint64_t       uint64;

#ifdef BWC_SINGLE_PRECISION
typedef float          bwc_float;
typedef uint32         bwc_raw;
#define PREC_BIT            31
#define MAXIMUM_NO_PASSES   ((32 * 3) - 2)
#else
typedef double         bwc_float;
typedef uint64         bwc_raw;
#define PREC_BIT            63
#define MAXIMUM_NO_PASSES   ((64 * 3) - 2)
#endif

/* ---- enumerations (constants.h:60-117) ---------------------------------------------------- */
typedef enum { bwc_dwt_9_7, bwc_dwt_5_3, bwc_dwt_haar } bwc_dwt_filter;
typedef enum { bwc_prog_LRCP, bwc_prog_RLCP, bwc_prog_RPCL, bwc_prog_PCRL, bwc_prog_CPRL } bwc_prog_ord;
typedef enum { bwc_qt_none, bwc_qt_derived } bwc_quant_st;
typedef enum { bwc_tile_sizeof, bwc_tile_numbof } bwc_tile_instr;
typedef enum
{
  bwc_precision_half   = 2,
  bwc_precision_single = 4,
  bwc_precision_double = 8
} bwc_precision;
typedef enum { comp, decomp } bwc_mode;

/* ---- user-visible structs (types.h) -------------------------------------------------------- */
typedef struct                      /* types.h:89-96 */
{
  uint64  size;
  uint64  position;
  uchar  *access;
  uchar  *memory;
} bwc_span;

typedef struct                      /* types.h:137-146 */
{
  uint64        nX, nY, nZ;
  uint64        nTS;
  uint8         nPar;
  bwc_precision data_prec;
  bwc_precision codec_prec;
} bwc_gl_inf;

typedef struct                      /* types.h:155-167 */
{
  struct codestream
  {
    bwc_span *aux;
    bwc_span *com;
  } codestream;
  void     *inp;
  void     *out;
  bwc_mode  mode;
} bwc_stream;

typedef struct                      /* types.h:532-570 */
{
  uint16         CSsgc;
  uchar          error_resilience;
  uint64         tileSizeX, tileSizeY;
  uint64         tileSizeZ, tileSizeTS;
  uint64         nTiles;
  uint8          precSizeX, precSizeY;
  uint8          precSizeZ, precSizeTS;
  uint8          cbX, cbY;
  uint8          cbZ, cbTS;
  bwc_dwt_filter KernelX, KernelY;
  bwc_dwt_filter KernelZ, KernelTS;
  uint8          decompX, decompY;
  uint8          decompZ, decompTS;
  uint8          nDecomp;
  uint32         qt_exponent, qt_mantissa;
  uint8          Qm;
  float         *bitrate;
  uint8          nLayers;
  uint8          useLayer;
  uint8          guard_bits;
  uint64         headerSize;
  uint64         codestreamSize;
  bwc_quant_st   quantization_style;
  bwc_prog_ord   progression;
} bwc_gl_ctrl;

typedef struct                      /* types.h:578-584 */
{
  bwc_gl_inf  info;
  bwc_gl_ctrl control;
  bwc_span    aux;
  bwc_span    com;
} bwc_header;

struct bwc_b200_engine;             /* opaque codec state of this library */

typedef struct                      /* types.h:592-600; `tile` is opaque here */
{
  bwc_gl_inf              info;
  bwc_gl_ctrl             control;
  struct bwc_b200_engine *tile;
  bwc_mode                mode;
} bwc_codec;

/* ---- API (libbwc.h:67-161) ----------------------------------------------------------------- */
bwc_stream *bwc_init_stream(void *const inpbuf, void *const outbuf, bwc_mode const mode);
uchar       bwc_set_com(bwc_stream *const stream, char const *const com, uint16 const size);
uchar       bwc_set_aux(bwc_stream *const stream, char const *const aux, uint32 const size);
uchar       create_codec(bwc_codec *const codec);
bwc_codec  *configure_codec(bwc_codec *const codec, uint64 const nX, uint64 const nY,
                            uint64 const nZ, uint64 const nTS, uint8 const nPar,
                            bwc_precision const prec);
bwc_codec  *bwc_alloc_coder(uint64 const nX, uint64 const nY, uint64 const nZ,
                            uint64 const nTS, uint8 const nPar, bwc_precision const prec);
bwc_codec  *bwc_alloc_decoder(void);
void        bwc_free_codec(bwc_codec *const codec);
void        bwc_set_error_resilience(bwc_codec *const codec);
void        set_quant_style(bwc_codec *const codec, bwc_quant_st const quantization_style);
void        set_quant_step_size(bwc_codec *const codec, double const delta);
void        set_progression(bwc_codec *const codec, bwc_prog_ord const progression);
void        set_kernels(bwc_codec *const codec, bwc_dwt_filter const KernelX,
                        bwc_dwt_filter const KernelY, bwc_dwt_filter const KernelZ,
                        bwc_dwt_filter const KernelTS);
void        bwc_set_decomp(bwc_codec *const codec, uint8 const decompX, uint8 const decompY,
                           uint8 const decompZ, uint8 const decompTS);
void        bwc_set_precincts(bwc_codec *const codec, uint8 const pX, uint8 const pY,
                              uint8 const pZ, uint8 const pTS);
void        bwc_set_codeblocks(bwc_codec *const codec, uint8 const cbX, uint8 const cbY,
                               uint8 const cbZ, uint8 const cbTS);
void        bwc_set_qm(bwc_codec *const codec, uint8 const Qm);
void        bwc_set_tiles(bwc_codec *const codec, uint64 const tilesX, uint64 const tilesY,
                          uint64 const tilesZ, uint64 const tilesTS, bwc_tile_instr const instr);
bwc_header *bwc_open_header(void *const inpbuf);
void        bwc_close_header(bwc_header *const header);
uchar       bwc_create_compression(bwc_codec *const codec, bwc_stream *const data,
                                   char *const rate_control);
size_t      bwc_compress(bwc_codec *const codec, bwc_stream *const data);
uchar       bwc_create_decompression(bwc_codec *const codec, bwc_stream *const stream,
                                     uint8 const layer);
uchar       bwc_decompress(bwc_codec *const codec, bwc_stream *const stream);

#ifdef __cplusplus
}
#endif

#endif /* BWC_H */
