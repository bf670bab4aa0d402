// Tier-1 decoding of one codeblock: the sequential decoder (one lane) and the dequantisation
// (a warp), shared by the CUDA kernel and the host build of the kernel bodies.
//
// Reference: decoding passes (tier1.c:1543-2069), decode_codeblock (tier1.c:2624-2787), MQ
// decoder (mq.c:147-173 fill_lsb, :846-919 initialize_mq_decoder, :950-1029 mq_bit_decode),
// dequantisation cblkcopy_inverse (tier1.c:767-931).
//
// Decoding is sequential inside a codeblock: every context depends on the decisions just made.
// The state lives as 64-bit sample masks per group of 16 stripe columns (bit 4i + r = row r of
// column i, as in the encoder's modelling kernel): significance, sign, visited in the current
// significance pass, refined, and the current plane's decoded bits, in shared memory.  One lane
// walks the passes group by group, holding the group's masks in registers; the neighbourhood of
// a column is cut from them (left and right columns, rows above and below) and from the other
// groups' masks (the stripes above and below).  Because groups are written back in scan order,
// the shared masks show earlier groups after the pass and later ones before it, exactly what
// the reference's in-place state shows.  Contexts come from two 256-entry tables built per
// codeblock class: significance context by (left rows r-1..r+1, right rows r-1..r+1, own rows
// r-1 and r+1), sign context and flip by the horizontal and vertical significance and sign bits.
// Decoded bits go to one mask per group and plane in global memory, written once per plane; the
// warp then rebuilds the magnitudes from those masks (8x8 bit transposes) and dequantises.
#pragma once

#include "t1_model.cuh"
#include "t1_mq.cuh"

namespace bwcb {
namespace t1 {

// per-codeblock-class tables: significance context index (0..8, before kCtxSig) and sign
// context | flip << 7
struct DecTables {
  uint8_t sigctx[3][256];
  uint8_t signctx[256];
};

// index of the significance-context table: rows r-1, r, r+1 of the left and right columns
// (3 bits each) and rows r-1, r+1 of the own column (2 bits)
T1_HD uint32_t sig_index_of(uint32_t l3, uint32_t r3, uint32_t o2) { return l3 | (r3 << 3) | (o2 << 6); }

// fills the tables from the format's 45-entry significance map and sign tables
T1_HD void dec_table_entry(DecTables &t, int i, const uint8_t *sig2ctx_all, const uint8_t *sig2xi,
                           const uint8_t *xi2cont) {
  // i in [0, 256)
  const uint32_t l3 = i & 7, r3 = (i >> 3) & 7, o2 = (i >> 6) & 3;
  const uint32_t h = ((l3 >> 1) & 1) + ((r3 >> 1) & 1);
  const uint32_t v = (o2 & 1) + ((o2 >> 1) & 1);
  const uint32_t d = (l3 & 1) + ((l3 >> 2) & 1) + (r3 & 1) + ((r3 >> 2) & 1);
  for (int cls = 0; cls < 3; ++cls) t.sigctx[cls][i] = sig2ctx_all[cls * 45 + 15 * h + 5 * v + d];
  // sign: xh = Lsig | Rsig << 1 | Lsign << 2 | Rsign << 3, xv likewise (above, below)
  const uint32_t xh = i & 15, xv = (i >> 4) & 15;
  t.signctx[i] = xi2cont[(sig2xi[xh] << 2) | sig2xi[xv]];
}

// ---- MQ decoder ---------------------------------------------------------------------------------

struct MqDec {
  uint32_t A, C, T;
  int32_t t;
  uint32_t L, Lmax;
  const uint8_t *b;    // the codeblock's bytes, 16-byte aligned, readable 32 bytes past Lmax
  Chunk cur, nxt;      // chunk L >> 4 and the one after it
  uint32_t cidx;
};

// byte i of a chunk (selects, so the chunk stays in registers)
T1_HD uint32_t chunk_byte(const Chunk &c, uint32_t i) {
  const uint32_t lo = (i & 4u) ? c.w[1] : c.w[0], hi = (i & 4u) ? c.w[3] : c.w[2];
  return (((i & 8u) ? hi : lo) >> (8 * (i & 3u))) & 0xFFu;
}

T1_HD uint32_t dec_byte(MqDec &d, uint32_t L) {
  if ((L >> 4) != d.cidx) {
    if ((L >> 4) == d.cidx + 1) {
      d.cur = d.nxt;
    } else {
      d.cur = load_chunk(d.b + (L & ~15u));
    }
    d.cidx = L >> 4;
    d.nxt = load_chunk(d.b + 16ull * (d.cidx + 1));
  }
  return chunk_byte(d.cur, L & 15u);
}

// fill_lsb (mq.c:147-173): the next byte into C, or 0xFF past the end / at a marker
T1_HD void dec_fill(MqDec &d) {
  if (d.L == d.Lmax || (d.T == 0xFF && dec_byte(d, d.L) > 0x8F)) {
    d.t = 8;
    d.C += 0xFF;
  } else if (d.T == 0xFF) {
    d.t = 7;
    d.T = dec_byte(d, d.L);
    d.C += d.T << 1;
    d.L++;
  } else {
    d.t = 8;
    d.T = dec_byte(d, d.L);
    d.C += d.T;
    d.L++;
  }
}

T1_HD void dec_init(MqDec &d, const uint8_t *b, uint32_t Lmax) {
  d.b = b;
  d.Lmax = Lmax;
  d.L = 0;
  d.T = 0;
  d.C = 0;
  d.t = 0;
  d.A = 0;
  d.cidx = 0;
  d.cur = load_chunk(b);
  d.nxt = load_chunk(b + 16);
  dec_fill(d);
  d.C <<= 8;
  dec_fill(d);
  d.C <<= 7;
  d.t -= 7;
  d.A = 0x8000;
}

// renormalisation: shift A and C left until A >= 0x8000, reading the next byte whenever the
// bit counter is empty before a shift (done in runs between byte reads).  Not inlined: the
// decoder calls it from a dozen places, and its inlined copies (with the byte reads) made the
// decoding loop too large for the instruction cache (decoding at 512^3: 249 -> 226 ms).
static __host__ __device__ __noinline__ void dec_renorm(MqDec &d) {
  int sh = clz32(d.A) - 16;
  do {
    if (d.t == 0) dec_fill(d);
    const int s1 = sh < d.t ? sh : d.t;
    d.A = (d.A << s1) & 0xFFFFu;
    d.C <<= s1;
    d.t -= s1;
    sh -= s1;
  } while (sh > 0);
}

// mq_bit_decode (mq.c:950-1029); slot holds the context's full table entry
T1_HD uint32_t dec_bit(MqDec &d, uint32_t *slot, const uint32_t *tbl) {
  const uint32_t ent = *slot;
  const uint32_t qe = ent & 0xFFFFu, mps = (ent >> 16) & 1u;
  d.A = (d.A - qe) & 0xFFFFu;
  if ((d.C >> 8) >= qe) {
    d.C = (d.C - (qe << 8)) & 0xFFFFFFu;
    if (d.A & 0x8000u) return mps;
    const bool lps = d.A < qe;
    *slot = tbl[lps ? (ent >> 24) & 0x7F : (ent >> 17) & 0x7F];
    dec_renorm(d);
    return lps ? 1u - mps : mps;
  }
  const bool m = d.A < qe;
  *slot = tbl[m ? (ent >> 17) & 0x7F : (ent >> 24) & 0x7F];
  d.A = qe;
  dec_renorm(d);
  return m ? mps : 1u - mps;
}

// ---- the sequential decoder ----------------------------------------------------------------

// bit i set when nibble i of m is not zero
T1_HD uint32_t nib_any(u64 m) {
  m = (m | (m >> 1));
  m = (m | (m >> 2)) & kRow0;
  m = (m | (m >> 3)) & 0x0303030303030303ull;
  m = (m | (m >> 6)) & 0x000F000F000F000Full;
  m = (m | (m >> 12)) & 0x000000FF000000FFull;
  m = (m | (m >> 24)) & 0xFFFFull;
  return (uint32_t)m;
}

// bit i set when nibble i of m is all ones
T1_HD uint32_t nib_all(u64 m) { return ~nib_any(~m) & 0xFFFFu; }

struct DecOut {
  int bitplane;   // first plane not decoded completely (the reference's `bitplane`)
  int cpass;      // pass reached in it (0 when it was not started)
  int pmin;       // lowest plane any of whose decisions were decoded (K when none)
};

// Decodes Z passes of the codeblock's bytes into the masks sig/sgn/pi (per group, shared) and
// one decoded-bit mask per plane and group in planes[b * ngroups + g]; slot[19] are the
// contexts' state entries.  Geometry: W columns per stripe row, H rows, ncols stripe columns.
T1_HD DecOut decode_seq(const uint8_t *bytes, uint32_t Lmax, int K, int Z, bool erres,
                        uint32_t W, uint32_t H, uint32_t ncols, int cls, u64 *sig, u64 *sgn,
                        u64 *pi, u64 *del, u64 *bits, uint32_t *slot, const uint32_t *tbl,
                        const DecTables &tabs, u64 *planes) {
  const int ngroups = (int)((ncols + 15) >> 4);
  const uint32_t nstripes = (H + 3) >> 2, nfull = H >> 2, rem = H & 3;
  const uint8_t *sigctx = tabs.sigctx[cls];
  for (int g = 0; g < ngroups; ++g) {
    sig[g] = 0;
    sgn[g] = 0;
    pi[g] = 0;
    del[g] = 0;
    bits[g] = 0;
  }
  for (int k = 0; k < dev::kCtxTotal; ++k) slot[k] = tbl[dev::mq_initial_state(k)];
  DecOut res{0, 0, K};
  if (Z <= 0) return res;
  MqDec d;
  dec_init(d, bytes, Lmax);
  const int Wi = (int)W;
  const bool wide = W >= 16;   // the stripes above and below lie in other groups

  // significance nibble of any column as the scan sees it (current group from registers)
  auto nib = [&](const u64 *arr, u64 cur, int g, int col) -> uint32_t {
    if (col < 0 || col >= (int)ncols) return 0u;
    const int gg = col >> 4;
    const u64 m = (gg == g) ? cur : arr[gg];
    return (uint32_t)(m >> (4 * (col & 15))) & 0xFu;
  };

  int i = 2, j = Z, k = K;
  bool stop = false;
  while (k-- > 0) {
    const int b = k;
    for (; i < 3; ++i, --j) {
      if (j == 0) {
        stop = true;
        break;
      }
      if (b < res.pmin) res.pmin = b;
      const int kind = i;
      uint32_t gx = 0, gj = 0;   // cursor (x, stripe) of column 16g
      for (int g = 0; g < ngroups; ++g) {
        u64 S = sig[g], G = sgn[g], P = pi[g], D = del[g], Bt = bits[g];
        const int c0 = 16 * g;
        // valid samples of the group (rows below a partial last stripe do not exist)
        const uint32_t ncg = ((int)ncols - c0 < 16) ? (uint32_t)((int)ncols - c0) : 16u;
        u64 VALID = (ncg == 16) ? ~0ull : ((1ull << (4 * ncg)) - 1ull);
        if (rem) VALID = col_masks(g, W, nstripes, nfull, rem, ncols).valid;
        // the columns that can need a decision in this pass: significance propagation visits
        // insignificant samples next to significant ones (a column that becomes significant
        // adds its right neighbour below); refinement the significant, unvisited samples;
        // cleanup the insignificant, unvisited ones.  A group with none skips the neighbourhood.
        uint32_t work;
        uint32_t candcols = 0;
        if (kind == 0) work = candcols = nib_any(~S & VALID);
        else if (kind == 1) work = nib_any(S & ~P & VALID);
        else work = nib_any(~S & ~P & VALID);
        if (work) {
        // neighbours in other groups: left / right boundary columns, stripes above and below
        const uint32_t Lb = (g > 0) ? (uint32_t)(sig[g - 1] >> 60) : 0u;
        const uint32_t LbS = (g > 0) ? (uint32_t)(sgn[g - 1] >> 60) : 0u;
        const uint32_t Rb = (g + 1 < ngroups) ? (uint32_t)(sig[g + 1] & 0xF) : 0u;
        const uint32_t RbS = (g + 1 < ngroups) ? (uint32_t)(sgn[g + 1] & 0xF) : 0u;
        u64 Uw = 0, ULw = 0, URw = 0, Dw = 0, DLw = 0, DRw = 0, UsW = 0, DsW = 0;
        if (wide) {
          Uw = window(sig, c0 - Wi, ngroups);
          ULw = window(sig, c0 - Wi - 1, ngroups);
          URw = window(sig, c0 - Wi + 1, ngroups);
          Dw = window(sig, c0 + Wi, ngroups);
          DLw = window(sig, c0 + Wi - 1, ngroups);
          DRw = window(sig, c0 + Wi + 1, ngroups);
          UsW = window(sgn, c0 - Wi, ngroups);
          DsW = window(sgn, c0 + Wi, ngroups);
        }
        if (kind == 0 && wide) {
          const uint32_t sigcols = nib_any(S);
          const uint32_t ud = nib_any(((Uw | ULw | URw) & kRow3) | ((Dw | DLw | DRw) & kRow0));
          const uint32_t nbc = sigcols | (sigcols << 1) | (sigcols >> 1) | (Lb ? 1u : 0u) |
                               (Rb ? 0x8000u : 0u) | ud;
          work = candcols & nbc & 0xFFFFu;
        }
        // cleanup: a column of a full stripe with no significant or visited sample and nothing
        // significant around it (a superset of its neighbourhood: the columns before and after it
        // in scan order and the stripes above and below) starts with its run decision, and a 0
        // ends the column with its state unchanged, before any neighbourhood is cut out.  A
        // column that becomes significant takes the run start from the column after it.
        uint32_t runcols = 0;
        if (kind == 2 && wide) {
          const uint32_t sigcols = nib_any(S);
          const uint32_t busy = nib_any(S | P) | (sigcols << 1) | (sigcols >> 1) | (Lb ? 1u : 0u) |
                                (Rb ? 0x8000u : 0u) |
                                nib_any(((Uw | ULw | URw) & kRow3) | ((Dw | DLw | DRw) & kRow0));
          runcols = nib_all(VALID) & ~busy & work;
        }
        while (work) {
          const int ci = ctz64(work);
          work &= work - 1u;
          bool run_one = false;   // the column's run decision was decoded here, as a 1
          if ((runcols >> ci) & 1u) {
            if (!dec_bit(d, &slot[dev::kCtxRun], tbl)) continue;
            run_one = true;
          }
          const int col = c0 + ci;
          uint32_t x, js;
          if (wide) {
            x = gx + (uint32_t)ci;
            js = gj;
            if (x >= W) {
              x -= W;
              js = (gj + 1 == nstripes) ? 0u : gj + 1;
            }
          } else {
            const uint32_t xx = gx + (uint32_t)ci;
            x = xx % W;
            js = (gj + xx / W) % nstripes;
          }
          const uint32_t own0 = (uint32_t)(S >> (4 * ci)) & 0xFu;
          const bool full = js < nfull;
          const uint32_t rows = full ? 4u : rem;
          const uint32_t vm = (1u << rows) - 1u;
          const bool xl = x > 0, xr = x + 1 < W, hu = js > 0, hd = full && js + 1 < nstripes;
          const int sh = 4 * ci;
          uint32_t own = (uint32_t)(S >> sh) & 0xFu;
          const uint32_t opi = (uint32_t)(P >> sh) & 0xFu;
          // does this column need its neighbourhood?
          bool need;
          if (kind == 0) need = (own & vm) != vm;
          else if (kind == 1) need = ((own & ~opi & vm) & ~(uint32_t)(D >> sh)) != 0;
          else need = (~own & ~opi & vm) != 0;
          if (!need) {
            if (kind == 0) P &= ~(0xFull << sh);   // significant samples are not visited
            if (kind == 1) {
              // refinement of samples already refined before: context 17
              const uint32_t todo = own & ~opi & vm;
              for (uint32_t r = 0; r < 4; ++r) {
                if (!((todo >> r) & 1u)) continue;
                if (dec_bit(d, &slot[dev::kCtxMag + 2], tbl)) Bt |= 1ull << (sh + r);
              }
              D |= (u64)todo << sh;
            }
          } else {
            // neighbourhood: 6-row words (row -1 at bit 0, rows 0-3 at 1-4, row 4 at bit 5)
            uint32_t Ln, Rn, LnS, RnS, ul, u, ur, dl, dd, dr, us, ds;
            if (ci > 0) {
              Ln = (uint32_t)(S >> (sh - 4)) & 0xFu;
              LnS = (uint32_t)(G >> (sh - 4)) & 0xFu;
            } else {
              Ln = Lb;
              LnS = LbS;
            }
            if (ci < 15) {
              Rn = (uint32_t)(S >> (sh + 4)) & 0xFu;
              RnS = (uint32_t)(G >> (sh + 4)) & 0xFu;
            } else {
              Rn = Rb;
              RnS = RbS;
            }
            if (!xl) Ln = LnS = 0;
            if (!xr) Rn = RnS = 0;
            if (wide) {
              u = (uint32_t)(Uw >> (sh + 3)) & 1u;
              ul = (uint32_t)(ULw >> (sh + 3)) & 1u;
              ur = (uint32_t)(URw >> (sh + 3)) & 1u;
              us = (uint32_t)(UsW >> (sh + 3)) & 1u;
              dd = (uint32_t)(Dw >> sh) & 1u;
              dl = (uint32_t)(DLw >> sh) & 1u;
              dr = (uint32_t)(DRw >> sh) & 1u;
              ds = (uint32_t)(DsW >> sh) & 1u;
            } else {
              u = (nib(sig, S, g, col - Wi) >> 3) & 1u;
              ul = (nib(sig, S, g, col - Wi - 1) >> 3) & 1u;
              ur = (nib(sig, S, g, col - Wi + 1) >> 3) & 1u;
              us = (nib(sgn, G, g, col - Wi) >> 3) & 1u;
              dd = nib(sig, S, g, col + Wi) & 1u;
              dl = nib(sig, S, g, col + Wi - 1) & 1u;
              dr = nib(sig, S, g, col + Wi + 1) & 1u;
              ds = nib(sgn, G, g, col + Wi) & 1u;
            }
            if (!hu) u = ul = ur = us = 0;
            if (!hd) dd = dl = dr = ds = 0;
            if (!xl) ul = dl = 0;
            if (!xr) ur = dr = 0;
            const uint32_t Lx = ul | (Ln << 1) | (dl << 5), Rx = ur | (Rn << 1) | (dr << 5);
            const uint32_t LxS = (LnS << 1), RxS = (RnS << 1);
            uint32_t gown = (uint32_t)(G >> sh) & 0xFu;
            auto ctx_sig = [&](uint32_t r) -> uint32_t {
              const uint32_t Ox = u | (own << 1) | (dd << 5);
              const uint32_t o2 = ((Ox >> r) & 1u) | (((Ox >> (r + 2)) & 1u) << 1);
              return dev::kCtxSig + sigctx[sig_index_of((Lx >> r) & 7u, (Rx >> r) & 7u, o2)];
            };
            auto dec_sign = [&](uint32_t r) -> uint32_t {
              const uint32_t Ox = u | (own << 1) | (dd << 5);
              const uint32_t OxS = us | (gown << 1) | (ds << 5);
              const uint32_t xh = ((Lx >> (r + 1)) & 1u) | (((Rx >> (r + 1)) & 1u) << 1) |
                                  (((LxS >> (r + 1)) & 1u) << 2) | (((RxS >> (r + 1)) & 1u) << 3);
              const uint32_t xv = ((Ox >> r) & 1u) | (((Ox >> (r + 2)) & 1u) << 1) |
                                  (((OxS >> r) & 1u) << 2) | (((OxS >> (r + 2)) & 1u) << 3);
              const uint32_t e = tabs.signctx[xh | (xv << 4)];
              return dec_bit(d, &slot[e & 0x7Fu], tbl) ^ (e >> 7);
            };
            // a sample becomes significant: bit, sign, state
            auto set_sig = [&](uint32_t r) {
              Bt |= 1ull << (sh + r);
              const uint32_t sgnbit = dec_sign(r);
              gown |= sgnbit << r;
              G |= (u64)sgnbit << (sh + r);
              own |= 1u << r;
              S |= 1ull << (sh + r);
            };
            if (kind == 0) {
              uint32_t pv = 0;
              for (uint32_t r = 0; r < rows; ++r) {
                if ((own >> r) & 1u) continue;
                const uint32_t Ox = u | (own << 1) | (dd << 5);
                const uint32_t any = ((Lx >> r) & 7u) | ((Rx >> r) & 7u) | ((Ox >> r) & 5u);
                if (!any) continue;
                if (dec_bit(d, &slot[ctx_sig(r)], tbl)) set_sig(r);
                pv |= 1u << r;
              }
              P = (P & ~(0xFull << sh)) | ((u64)pv << sh);
            } else if (kind == 1) {
              const uint32_t todo = own & ~opi & vm;
              const uint32_t dn = (uint32_t)(D >> sh) & 0xFu;
              for (uint32_t r = 0; r < rows; ++r) {
                if (!((todo >> r) & 1u)) continue;
                uint32_t ctx;
                if ((dn >> r) & 1u) {
                  ctx = dev::kCtxMag + 2;
                } else {
                  const uint32_t Ox = u | (own << 1) | (dd << 5);
                  const uint32_t any = ((Lx >> r) & 7u) | ((Rx >> r) & 7u) | ((Ox >> r) & 5u);
                  ctx = dev::kCtxMag + (any ? 1u : 0u);
                }
                if (dec_bit(d, &slot[ctx], tbl)) Bt |= 1ull << (sh + r);
              }
              D |= (u64)todo << sh;
            } else {
              uint32_t r = 0;
              bool skip_first = false;
              if (full && own == 0 && opi == 0 && !(Lx | Rx | u | dd)) {
                // run mode (the run decision already decoded when run_one)
                if (!run_one && !dec_bit(d, &slot[dev::kCtxRun], tbl)) {
                  r = 4;
                } else {
                  r = dec_bit(d, &slot[dev::kCtxUni], tbl) << 1;
                  r |= dec_bit(d, &slot[dev::kCtxUni], tbl);
                  skip_first = true;
                }
              }
              for (; r < rows; ++r) {
                if (((own | opi) >> r) & 1u) continue;
                uint32_t bit;
                if (skip_first) {
                  skip_first = false;
                  bit = 1;
                } else {
                  bit = dec_bit(d, &slot[ctx_sig(r)], tbl);
                }
                if (bit) set_sig(r);
              }
            }
          }
          if (kind == 0 && ci < 15 && (((uint32_t)(S >> (4 * ci)) & 0xFu) != own0))
            work |= candcols & (2u << ci);   // the right neighbour may now be visited
          if (kind == 2 && (((uint32_t)(S >> (4 * ci)) & 0xFu) != own0))
            runcols &= ~(2u << ci);   // its right neighbour has a significant neighbour now
        }
        }   // work
        // cursor of the next group
        gx += 16;
        while (gx >= W) {
          gx -= W;
          if (++gj == nstripes) gj = 0;
        }
        if (kind == 2) {
          // the plane's decoded bits are final; the next significance pass starts unvisited
          planes[(uint64_t)b * ngroups + g] = Bt;
          Bt = 0;
          P = 0;
        }
        sig[g] = S;
        sgn[g] = G;
        pi[g] = P;
        del[g] = D;
        bits[g] = Bt;
      }
    }
    if (stop) break;
    if (erres) {
      uint32_t v = dec_bit(d, &slot[dev::kCtxUni], tbl) << 3;
      v |= dec_bit(d, &slot[dev::kCtxUni], tbl) << 2;
      v |= dec_bit(d, &slot[dev::kCtxUni], tbl) << 1;
      v |= dec_bit(d, &slot[dev::kCtxUni], tbl);
      if (v != 0x0A) {
        stop = true;
        break;
      }
    }
    i = 0;
  }
  if (!stop) i = 0;
  res.bitplane = (k > 0) ? k : 0;
  res.cpass = i;
  // a plane whose cleanup pass was not reached keeps its decoded bits in `bits`
  if (res.pmin < K && i > 0 && i < 3) {
    for (int g = 0; g < ngroups; ++g) planes[(uint64_t)res.bitplane * ngroups + g] = bits[g];
  }
  return res;
}

// Dequantisation of group g's 64 samples (tier1.c:895-910): value = (m + 0.475 * 2^p) * step
// with p the first undecoded plane (one higher for samples the interrupted significance pass
// did not visit) and the decoded sign; zero magnitudes are left as they are (zero).
T1_HD void dequant_group(int g, int ngroups, int K, const DecOut &res, const u64 *planes,
                         u64 sgnm, u64 pim, const CbDev &cb, bwc_float qt_eff, bwc_float *work,
                         uint32_t W, uint32_t H, uint32_t ncols) {
  if (res.pmin >= K) return;
  const uint32_t nstripes = (H + 3) >> 2, nfull = H >> 2, rem = H & 3;
  const uint32_t c0 = 16u * (uint32_t)g;
  uint32_t x = c0 % W;
  uint32_t sr = c0 / W;
  uint32_t js = sr % nstripes, sl = sr / nstripes;
  const int g0 = res.pmin >> 3, g1 = (K - 1) >> 3;
#pragma unroll 1
  for (int pair = 0; pair < 8; ++pair) {
    bwc_raw q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int gb = g0; gb <= g1; ++gb) {
      u64 m = 0;
      for (int jb = 0; jb < 8; ++jb) {
        const int b = 8 * gb + jb;
        if (b < res.pmin || b >= K) continue;
        const u64 pm = planes[(uint64_t)b * ngroups + g];
        m |= ((pm >> (8 * pair)) & 0xFFull) << (8 * jb);
      }
      m = transpose8(m);   // byte s: sample s's bits of planes 8gb .. 8gb+7
      for (int s = 0; s < 8; ++s) q[s] |= (bwc_raw)((m >> (8 * s)) & 0xFFull) << (8 * gb);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t ci = 2u * pair + h;
      const uint32_t col = c0 + ci;
      if (col < ncols) {
        const uint32_t rows = (js < nfull) ? 4u : rem;
#pragma unroll
        for (uint32_t r = 0; r < 4; ++r) {
          const bwc_raw m = q[4 * h + r];
          if (r >= rows || !m) continue;
          const int p = 4 * ci + r;
          const int visited = (int)((pim >> p) & 1ull);
          const int shift = res.bitplane + ((!res.cpass || visited) ? 0 : 1);
#ifdef __CUDA_ARCH__
          const float off = __fmul_rn((float)((uint64_t)1 << shift), 0.475f);
          bwc_float f = dev::from_u64_rn((uint64_t)m);
          f = dev::fadd(f, (bwc_float)off);
          f = dev::fmul(f, qt_eff);
#else
          const float off = (float)((uint64_t)1 << shift) * 0.475f;
          bwc_float f = (bwc_float)(uint64_t)m;
          f = f + (bwc_float)off;
          f = f * qt_eff;
#endif
          const bwc_raw rr = raw_of(f) | (((sgnm >> p) & 1ull) ? kSignMask : (bwc_raw)0);
          const uint32_t y = 4 * js + r, z = sl % cb.d, tt = sl / cb.d;
          work[cb.base + (uint64_t)(cb.x0 + x) + (uint64_t)(cb.y0 + y) * cb.sy +
               (uint64_t)(cb.z0 + z) * cb.sz + (uint64_t)(cb.t0 + tt) * cb.st] = float_of(rr);
        }
      }
      if (++x == W) {
        x = 0;
        if (++js == nstripes) {
          js = 0;
          ++sl;
        }
      }
    }
  }
}

}  // namespace t1
}  // namespace bwcb
