/*
 * ref_probe.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin stage-by-stage driver around the unmodified reference library (BigWhoop libbwc),
 * compiled into the same shared object as the reference sources by oracle/Makefile.  It lets
 * the parity tests stop the reference after any stage of its compression path and read the
 * intermediate results (normalised field, wavelet coefficients, per-codeblock tier-1 output,
 * codestream), and reset the reference's process-global wavelet energy-gain table.
 *
 * Nothing in the product library links to or calls this file.
 *
 * The stage order follows bwc_compress (src/library/libbwc.c:3145-3438) and bwc_decompress
 * (src/library/libbwc.c:3485-3710).  fill_buffer, normalize_param, denormalize_param and
 * flush_buffer are `static` in libbwc.c, so the four helpers below restate them
 * (libbwc.c:622-812, :993-1078, :1093-1176, :827-978) with the same arithmetic.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#if defined(_OPENMP)
#include <omp.h>
#endif

#include "libbwc.h"
#include "dwt.h"
#include "tier1.h"
#include "tier2.h"
#include "codestream.h"

typedef struct
{
   bwc_codec  *codec;
   bwc_stream *stream;
   bwc_sample *work;       /* working buffer of one tile/parameter */
   uint64      work_len;
   char       *rate;       /* private copy: the reference tokenises it in place */
   int         tile;       /* the tile the stage functions work on (rp_select_tile) */
} rp_handle;

/* ---- configuration ------------------------------------------------------------------- */

int rp_prec_bytes(void) { return PREC_BYTE; }

void rp_set_threads(int n)
{
#if defined(_OPENMP)
   if(n > 0) omp_set_num_threads(n);
#else
   (void)n;
#endif
}

int rp_max_threads(void)
{
#if defined(_OPENMP)
   return omp_get_max_threads();
#else
   return 1;
#endif
}

/* Zero the reference's global DWT_ENERGY_GAIN_LUT (dwt.c:80): every initialize_gain_lut call
 * adds to it, so the tests bring it back to its load-time state before comparing. */
void rp_reset_gain_lut(void)
{
   memset(DWT_ENERGY_GAIN_LUT, 0, sizeof(DWT_ENERGY_GAIN_LUT));
}

void rp_get_gain_lut(double *out)
{
   memcpy(out, DWT_ENERGY_GAIN_LUT, sizeof(DWT_ENERGY_GAIN_LUT));
}

/* ---- compression ----------------------------------------------------------------------- */

/* decomp/cb: 4 entries each or NULL (library defaults); qm < 0: default; erres: call
 * bwc_set_error_resilience once; rate NULL: lossless default (PREC_BIT + 1 bpv). */
/* precinct sizes (log2 per axis) applied by the next rp_open_compress calls; NULL: defaults */
static uint8 rp_prec[4];
static int   rp_prec_set = 0;
void rp_set_precincts(const uint8 *p)
{
   if(p) { memcpy(rp_prec, p, 4); rp_prec_set = 1; }
   else  rp_prec_set = 0;
}

/* wavelet kernels per axis (bwc_dwt_filter values) applied by the next rp_open_compress calls;
 * NULL: defaults (CDF 9/7) */
static uint8 rp_kern[4];
static int   rp_kern_set = 0;
void rp_set_kernels(const uint8 *k)
{
   if(k) { memcpy(rp_kern, k, 4); rp_kern_set = 1; }
   else  rp_kern_set = 0;
}

/* tile sizes per axis (bwc_set_tiles, bwc_tile_sizeof) applied by the next rp_open_compress
 * calls; NULL: one tile */
static uint64 rp_tiles[4];
static int    rp_tiles_set = 0;
void rp_set_tiles(const uint64 *t)
{
   if(t) { memcpy(rp_tiles, t, sizeof(rp_tiles)); rp_tiles_set = 1; }
   else  rp_tiles_set = 0;
}

/* stage functions below work on tile t (0 until selected) */
int rp_select_tile(rp_handle *h, int t)
{
   if(t < 0 || (uint64)t >= h->codec->control.nTiles) return 1;
   h->tile = t;
   return 0;
}

uint64 rp_num_tiles(rp_handle *h) { return h->codec->control.nTiles; }

rp_handle *rp_open_compress(void *field, uint64 nX, uint64 nY, uint64 nZ, uint64 nTS,
                            uint8 nPar, int data_prec, const uint8 *decomp, const uint8 *cb,
                            int qm, int erres, const char *rate, void *out)
{
   rp_handle *h = calloc(1, sizeof(rp_handle));
   if(!h) return NULL;
   h->codec = bwc_alloc_coder(nX, nY, nZ, nTS, nPar, (bwc_precision)data_prec);
   if(!h->codec) { free(h); return NULL; }
   if(erres)  bwc_set_error_resilience(h->codec);
   if(decomp) bwc_set_decomp(h->codec, decomp[0], decomp[1], decomp[2], decomp[3]);
   if(cb)     bwc_set_codeblocks(h->codec, cb[0], cb[1], cb[2], cb[3]);
   if(rp_prec_set) bwc_set_precincts(h->codec, rp_prec[0], rp_prec[1], rp_prec[2], rp_prec[3]);
   if(rp_tiles_set) bwc_set_tiles(h->codec, rp_tiles[0], rp_tiles[1], rp_tiles[2], rp_tiles[3],
                                  bwc_tile_sizeof);
   if(rp_kern_set) set_kernels(h->codec, (bwc_dwt_filter)rp_kern[0], (bwc_dwt_filter)rp_kern[1],
                               (bwc_dwt_filter)rp_kern[2], (bwc_dwt_filter)rp_kern[3]);
   if(qm >= 0) bwc_set_qm(h->codec, (uint8)qm);
   h->stream = bwc_init_stream(field, out, comp);
   if(rate)
   {
      h->rate = malloc(strlen(rate) + 1);
      strcpy(h->rate, rate);
   }
   if(bwc_create_compression(h->codec, h->stream, h->rate))
   {
      bwc_free_codec(h->codec);
      free(h->stream); free(h->rate); free(h);
      return NULL;
   }
   return h;
}

size_t rp_compress_full(rp_handle *h)
{
   return bwc_compress(h->codec, h->stream);
}

/* restatement of fill_buffer (libbwc.c:622-812) for the selected tile */
static void rp_fill(rp_handle *h, bwc_parameter *parameter, uint16 param_id)
{
   bwc_gl_inf    *info = &h->codec->info;
   bwc_tile_inf  *tile_info = &h->codec->tile[h->tile].info;
   bwc_param_inf *pi = &parameter->info;
   uint64 width  = pi->X1 - pi->X0, height = pi->Y1 - pi->Y0;
   uint64 depth  = pi->Z1 - pi->Z0, dt     = pi->TS1 - pi->TS0;
   uint64 off    = info->nX * info->nY * info->nZ * info->nTS * param_id;
   bwc_float mx = pi->parameter_max, mn = pi->parameter_min;
   uint64 x, y, z, t;
   parameter->data = h->work;
   for(t = 0; t < dt; ++t)
      for(z = 0; z < depth; ++z)
         for(y = 0; y < height; ++y)
         {
            uint64 s = off + tile_info->X0 + info->nX * (tile_info->Y0 + y + info->nY * (tile_info->Z0 + z + info->nZ * t));
            bwc_sample *d = &h->work[width * (y + height * (z + depth * t))];
            for(x = 0; x < width; ++x)
            {
               if(info->data_prec == bwc_precision_double)
                  d[x].f = (bwc_float)((double *)h->stream->inp)[s + x];
               else
                  d[x].f = (bwc_float)((float *)h->stream->inp)[s + x];
               mx = MAX(mx, d[x].f);
               mn = MIN(mn, d[x].f);
            }
         }
   pi->parameter_max = mx;
   pi->parameter_min = mn;
   parameter->control.alpha = (pi->parameter_max + pi->parameter_min) / 2.0f;
   parameter->control.beta  = 2.0f / (pi->parameter_max - pi->parameter_min);
}

/* restatement of normalize_param (libbwc.c:993-1078) */
static void rp_normalize(rp_handle *h, bwc_parameter *parameter)
{
   bwc_param_inf *pi = &parameter->info;
   uint64 n = (pi->X1 - pi->X0) * (pi->Y1 - pi->Y0) * (pi->Z1 - pi->Z0) * (pi->TS1 - pi->TS0);
   bwc_raw shift = (uint64)h->codec->control.Qm << PREC_MANTISSA;
   bwc_float alpha = parameter->control.alpha, beta = parameter->control.beta;
   uint64 x;
   for(x = 0; x < n; ++x)
   {
      bwc_sample *s = &parameter->data[x];
      s->f = (bwc_float)(s->f - alpha) * beta;
      s->raw += (((s->raw & EXPONENT) == 0) && ((s->raw & MANTISSA) == 0)) ? 0 : shift;
   }
}

static int rp_ensure_work(rp_handle *h)
{
   bwc_gl_ctrl *c = &h->codec->control;
   uint64 n = c->tileSizeX * c->tileSizeY * c->tileSizeZ * c->tileSizeTS;
   if(!h->work)
   {
      h->work = calloc(n, sizeof(bwc_sample));
      h->work_len = n;
   }
   return h->work ? 0 : 1;
}

/* fill + normalise parameter p of the selected tile into the working buffer */
int rp_stage_normalize(rp_handle *h, int p)
{
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   if(rp_ensure_work(h)) return 1;
   memset(h->work, 0, h->work_len * sizeof(bwc_sample));
   rp_fill(h, parameter, (uint16)p);
   rp_normalize(h, parameter);
   return 0;
}

int rp_stage_dwt(rp_handle *h, int p)
{
   return forward_wavelet_transform(h->codec, &h->codec->tile[h->tile].parameter[p]);
}

int rp_stage_t1(rp_handle *h, int p)
{
   return t1_encode(h->codec, &h->codec->tile[h->tile], &h->codec->tile[h->tile].parameter[p]);
}

int rp_stage_t2(rp_handle *h)
{
   return t2_encode(h->codec, &h->codec->tile[h->tile]);
}

size_t rp_stage_assemble(rp_handle *h)
{
   return assemble_codestream(h->codec, h->stream);
}

/* raw bytes of the working buffer (PREC_BYTE per value) */
uint64 rp_copy_work(rp_handle *h, void *dst)
{
   memcpy(dst, h->work, h->work_len * sizeof(bwc_sample));
   return h->work_len;
}

/* overwrite the first n values of the working buffer (PREC_BYTE per value); 1 if n exceeds it */
int rp_set_work(rp_handle *h, const void *src, uint64 n)
{
   if(rp_ensure_work(h) || n > h->work_len) return 1;
   memcpy(h->work, src, n * sizeof(bwc_sample));
   return 0;
}

/* parameter statistics after fill: min, max, alpha, beta (as double) */
void rp_param_stats(rp_handle *h, int p, double *out4)
{
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   out4[0] = parameter->info.parameter_min;
   out4[1] = parameter->info.parameter_max;
   out4[2] = parameter->control.alpha;
   out4[3] = parameter->control.beta;
}

uint64 rp_num_codeblocks(rp_handle *h, int p)
{
   return h->codec->tile[h->tile].parameter[p].control.number_of_codeblocks;
}

/* Codeblock c (tier-1 order) of parameter p:
 * geom[0..7] = X0,Y0,Z0,TS0,X1,Y1,Z1,TS1 (working-buffer coordinates), geom[8] = subband
 * highband flag, geom[9] = subband Kmax;
 * meta[0] = K, meta[1] = Kmsbs, meta[2] = Z;  L[0..Z-1], S[0..Z], data (L[Z-1] bytes). */
int rp_codeblock(rp_handle *h, int p, uint64 c, uint64 *geom, int64 *meta, uint64 *L,
                 uint16 *S, uint8 *data, uint64 cap)
{
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   bwc_cblk_access *a;
   bwc_encoded_cblk *e;
   uint64 n;
   if(c >= parameter->control.number_of_codeblocks) return 1;
   a = &parameter->access[c];
   e = a->codeblock->encoded_block;
   if(geom)
   {
      bwc_cblk_inf *ci = &a->codeblock->info;
      geom[0] = ci->X0; geom[1] = ci->Y0; geom[2] = ci->Z0; geom[3] = ci->TS0;
      geom[4] = ci->X1; geom[5] = ci->Y1; geom[6] = ci->Z1; geom[7] = ci->TS1;
      geom[8] = a->subband->control.highband_flag;
      geom[9] = a->subband->control.Kmax;
   }
   if(meta)
   {
      meta[0] = e->K; meta[1] = e->Kmsbs; meta[2] = e->Z;
   }
   if(L) memcpy(L, e->L, sizeof(e->L));
   if(S) memcpy(S, e->S, sizeof(e->S));
   if(data && e->data && e->Z > 0)
   {
      n = e->L[e->Z - 1];
      if(n > cap) return 2;
      memcpy(data, e->data, n);
   }
   return 0;
}

/* subband control of the subband holding codeblock c: qt_effective_step_size, qt_step_size,
 * dwt_gain (as double) */
void rp_codeblock_subband(rp_handle *h, int p, uint64 c, double *out3)
{
   bwc_cblk_access *a = &h->codec->tile[h->tile].parameter[p].access[c];
   out3[0] = a->subband->control.qt_effective_step_size;
   out3[1] = a->subband->control.qt_step_size;
   out3[2] = a->subband->info.dwt_gain;
}

void rp_tile_slopes(rp_handle *h, uint16 *out2)
{
   out2[0] = h->codec->tile[h->tile].control.slope_min;
   out2[1] = h->codec->tile[h->tile].control.slope_max;
}

/* copy of the public part of the codec: info and control (bitrate pointer excluded) */
void rp_codec_control(rp_handle *h, uint64 *out)
{
   bwc_gl_ctrl *c = &h->codec->control;
   out[0]  = c->CSsgc;       out[1]  = c->error_resilience;
   out[2]  = c->tileSizeX;   out[3]  = c->tileSizeY;  out[4] = c->tileSizeZ;  out[5] = c->tileSizeTS;
   out[6]  = c->nTiles;
   out[7]  = c->precSizeX;   out[8]  = c->precSizeY;  out[9] = c->precSizeZ;  out[10] = c->precSizeTS;
   out[11] = c->cbX;         out[12] = c->cbY;        out[13] = c->cbZ;       out[14] = c->cbTS;
   out[15] = c->decompX;     out[16] = c->decompY;    out[17] = c->decompZ;   out[18] = c->decompTS;
   out[19] = c->nDecomp;     out[20] = c->qt_exponent; out[21] = c->qt_mantissa; out[22] = c->Qm;
   out[23] = c->nLayers;     out[24] = c->guard_bits; out[25] = c->headerSize; out[26] = c->codestreamSize;
   out[27] = c->quantization_style; out[28] = c->progression;
}

void rp_close(rp_handle *h)
{
   if(!h) return;
   bwc_free_codec(h->codec);
   if(h->stream)
   {
      if(h->stream->codestream.aux) { free(h->stream->codestream.aux->memory); free(h->stream->codestream.aux); }
      if(h->stream->codestream.com) { free(h->stream->codestream.com->memory); free(h->stream->codestream.com); }
      free(h->stream);
   }
   free(h->work);
   free(h->rate);
   free(h);
}

/* ---- decompression --------------------------------------------------------------------- */

rp_handle *rp_open_decompress(void *codestream, void *out, uint8 layer)
{
   rp_handle *h = calloc(1, sizeof(rp_handle));
   if(!h) return NULL;
   h->codec = bwc_alloc_decoder();
   h->stream = bwc_init_stream(codestream, out, decomp);
   if(bwc_create_decompression(h->codec, h->stream, layer))
   {
      free(h->stream); free(h);
      return NULL;
   }
   return h;
}

int rp_decompress_full(rp_handle *h)
{
   return bwc_decompress(h->codec, h->stream);
}

int rp_dstage_t1(rp_handle *h, int p)
{
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   if(rp_ensure_work(h)) return 1;
   memset(h->work, 0, h->work_len * sizeof(bwc_sample));
   parameter->data = h->work;
   return t1_decode(h->codec, &h->codec->tile[h->tile], parameter);
}

int rp_dstage_idwt(rp_handle *h, int p)
{
   return inverse_wavelet_transform(h->codec, &h->codec->tile[h->tile].parameter[p]);
}

/* restatement of denormalize_param (libbwc.c:1093-1176) and flush_buffer (:827-978) */
int rp_dstage_finish(rp_handle *h, int p)
{
   bwc_gl_inf    *info = &h->codec->info;
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   bwc_param_inf *pi = &parameter->info;
   uint64 width  = pi->X1 - pi->X0, height = pi->Y1 - pi->Y0;
   uint64 depth  = pi->Z1 - pi->Z0, dt     = pi->TS1 - pi->TS0;
   uint64 n = width * height * depth * dt, x, y, z, t;
   uint64 off = info->nX * info->nY * info->nZ * info->nTS * p;
   bwc_raw shift = (uint64)h->codec->control.Qm << PREC_MANTISSA;
   bwc_float alpha = (pi->parameter_max + pi->parameter_min) / 2.0f;
   bwc_float beta  = (pi->parameter_max - pi->parameter_min) / 2.0f;
   for(x = 0; x < n; ++x)
   {
      bwc_sample *s = &parameter->data[x];
      s->raw -= (((s->raw & EXPONENT) == 0) && ((s->raw & MANTISSA) == 0)) ? 0 : shift;
      s->f = (bwc_float)(s->f * beta) + alpha;
   }
   for(t = 0; t < dt; ++t)
      for(z = 0; z < depth; ++z)
         for(y = 0; y < height; ++y)
         {
            uint64 d = off + pi->X0 + info->nX * (pi->Y0 + y + info->nY * (pi->Z0 + z + info->nZ * t));
            bwc_sample *s = &parameter->data[width * (y + height * (z + depth * t))];
            for(x = 0; x < width; ++x)
            {
               if(info->data_prec == bwc_precision_double)
                  ((double *)h->stream->out)[d + x] = (double)s[x].f;
               else
                  ((float *)h->stream->out)[d + x] = (float)s[x].f;
            }
         }
   return 0;
}

/* decoder-side codeblock state after parsing: meta[0] = K (Kmax - Kmsbs), [1] = Kmsbs, [2] = Z */
int rp_dcodeblock(rp_handle *h, int p, uint64 c, int64 *meta, uint64 *L)
{
   bwc_parameter *parameter = &h->codec->tile[h->tile].parameter[p];
   bwc_cblk_access *a;
   bwc_encoded_cblk *e;
   if(c >= parameter->control.number_of_codeblocks) return 1;
   a = &parameter->access[c];
   e = a->codeblock->encoded_block;
   meta[0] = a->subband->control.Kmax - e->Kmsbs;
   meta[1] = e->Kmsbs;
   meta[2] = e->Z;
   if(L) memcpy(L, e->L, sizeof(e->L));
   return 0;
}
