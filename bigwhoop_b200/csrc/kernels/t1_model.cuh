// Context modelling of one codeblock by a block of 256 threads: quantisation into bit planes,
// then every coding pass of every bit plane, each pass's decisions written (context << 1 |
// decision, one byte each) in the reference's scan order into the codeblock's symbol stream.
//
// Reference: cblkcopy_forward (tier1.c:526-729), significance propagation (tier1.c:962-1146),
// magnitude refinement (tier1.c:1177-1301), cleanup with run mode (tier1.c:1332-1511),
// distortion tables (tier1.c:139-165), segmentation symbols (tier1.c:94-100), the causal stripe
// neighbourhood (tier1.c:692-703).
//
// Layout.  Stripe columns are numbered in scan order, col = x + W * (stripe + stripes * slice).
// Thread t owns the 16 columns [16t, 16t + 16); its 64 samples are the bits of a 64-bit mask,
// bit 4i + r = row r of its column i, so ascending bit order is scan order, and the whole
// per-thread state is a handful of masks: significance, sign, visited in this plane's
// significance pass, refined at least once, and the bit planes.  Bit planes are stored in the
// codeblock's scratch as one 64-bit mask per thread and plane, written once after quantisation
// by 8x8 bit transposes.
//
// Neighbourhoods.  The neighbours of all 64 samples at once are shifted masks: the left and
// right columns are the thread's own mask shifted by one column (4 bits) plus the boundary
// column of the adjacent thread; the stripe above and below are 16-column windows cut from the
// published masks of the threads that own columns col -+ W.  Column-validity masks (x > 0,
// x < W-1, a stripe above in the same slice, a stripe below seen from row 3 of a full stripe)
// zero what does not exist.  Scan order decides which state a neighbour shows: samples scanned
// earlier (rows above in the column, the left column, the stripe above) show their state after
// the pass, later ones their state before it.
//
// Passes.
//  * significance propagation: a sample is visited when insignificant with a significant
//    neighbour, and becomes significant when visited with its bit set, so significance spreads
//    through the pass in scan order.  Each thread computes its columns' outcome in closed form
//    given the other threads' current estimates (iterating "outcome given neighbours" inside
//    its 64 samples to its least fixed point), publishes it, and the block repeats until no
//    estimate changes; dependencies point backwards in scan order and the outcome is monotone,
//    so this climbs to the sequential result.
//  * magnitude refinement: samples significant before the plane and not visited; all contexts
//    use the state after the significance pass.
//  * cleanup: samples neither significant nor visited; their state after the pass is known in
//    closed form (significant iff the bit is set); a full column whose four samples and whole
//    neighbourhood are insignificant is coded in run mode.
// Symbol and distortion counts come from popcounts; each thread writes its symbols into its
// place (block scan) of a shared-memory staging area, which is then copied to the pass's chunk
// of the stream with 16-byte stores.  Distortion decreases are sums over the coded samples of
// the reference's integer tables, which are linear in the magnitude bits below the plane, so
// they are popcounts of masked bit planes.
#pragma once

#include "t1_common.cuh"

namespace bwcb {
namespace t1 {

constexpr int kModelBlock = 256;
constexpr int kColsPerThread = 16;
constexpr uint32_t kModelMaxCols = (uint32_t)kModelBlock * kColsPerThread;   // 4096
constexpr u64 kRow0 = 0x1111111111111111ull;
constexpr u64 kRow3 = kRow0 << 3;
// staging of one pass: at most 10 decisions per column (cleanup in run mode: run, two position
// bits, a sign, and three samples of two) plus 4 segmentation symbols
constexpr uint32_t kStageBytes = 10 * kModelMaxCols + 16;

struct ModelShared {
  u64 sig[kModelBlock];       // published significance
  u64 fin[2][kModelBlock];    // post-pass estimates
  u64 sgn[kModelBlock];       // signs
  long long dsum[2];          // distortion sums (alternating passes)
  uint32_t wsum[kModelBlock / 32 + 1];
  uint32_t kmax;
  uint32_t ok;
  unsigned long long base;    // offset of the codeblock's stream in the arena
  uint8_t sig2ctx[48];
  uint8_t sig2xi[16];
  uint8_t xi2cont[16];
};

// bytes of scratch a codeblock of ncols stripe columns needs for its bit planes (one 64-bit
// mask per owning thread and plane)
T1_HD uint64_t model_plane_bytes(uint64_t ncols) {
  return ((ncols + 15) / 16) * 8ull * (uint64_t)(kPrecBit + 1);
}

struct ColMasks {
  u64 valid, xl, xr, hu, hd, full;
};

// validity masks of thread t's columns
T1_HD ColMasks col_masks(int t, uint32_t W, uint32_t nstripes, uint32_t nfull, uint32_t rem,
                         uint32_t ncols) {
  ColMasks m{0, 0, 0, 0, 0, 0};
  const uint32_t c0 = 16u * (uint32_t)t;
  if (c0 >= ncols) return m;
  uint32_t x = c0 % W, j = (c0 / W) % nstripes;
  for (int i = 0; i < 16; ++i) {
    if (c0 + i >= ncols) break;
    const bool full = j < nfull;
    const uint32_t rows = full ? 4u : rem;
    const u64 nib = 0xFull << (4 * i);
    m.valid |= (u64)((1u << rows) - 1u) << (4 * i);
    if (x > 0) m.xl |= nib;
    if (x + 1 < W) m.xr |= nib;
    if (j > 0) m.hu |= nib;
    if (full && j + 1 < nstripes) m.hd |= nib;
    if (full) m.full |= nib;
    if (++x == W) {
      x = 0;
      if (++j == nstripes) j = 0;
    }
  }
  return m;
}

// Columns [a, a + 16) of the per-thread masks m[] (thread k owns [16k, 16k + 16)); columns
// outside [0, 16 * nthr) read as zero.
T1_HD u64 window(const u64 *m, int a, int nthr) {
  if (a <= -16 || a >= 16 * nthr) return 0ull;
  const int ta = (a + 16 * kModelBlock) / 16 - kModelBlock;   // floor(a / 16)
  const int o = a - 16 * ta;
  const u64 lo = (ta >= 0) ? m[ta] : 0ull;
  if (o == 0) return lo;
  const u64 hi = (ta + 1 < nthr) ? m[ta + 1] : 0ull;
  return (lo >> (4 * o)) | (hi << (64 - 4 * o));
}

// significance of the eight neighbours of every sample: F = the thread's own state after the
// pass (rows above), S = before it (rows below); mP = everybody's state after the pass (left
// column, stripe above), mQ = before it (right column, stripe below)
struct Nb {
  u64 L, R, U, D, UL, UR, DL, DR;
  u64 Uext, Dext;   // the parts of U and D from the stripes above and below
};

T1_HD Nb neighbours(u64 F, u64 S, const u64 *mP, const u64 *mQ, int t, int nthr, int W,
                    const ColMasks &cm) {
  const int c0 = 16 * t;
  const u64 Lc = ((F << 4) | (t > 0 ? (mP[t - 1] >> 60) : 0ull)) & cm.xl;
  const u64 Rc = ((S >> 4) | (t + 1 < nthr ? (mQ[t + 1] << 60) : 0ull)) & cm.xr;
  Nb n;
  n.L = Lc;
  n.R = Rc;
  n.Uext = (window(mP, c0 - W, nthr) >> 3) & kRow0 & cm.hu;
  n.Dext = (window(mQ, c0 + W, nthr) << 3) & kRow3 & cm.hd;
  n.U = ((F << 1) & ~kRow0) | n.Uext;
  n.D = ((S >> 1) & ~kRow3) | n.Dext;
  n.UL = ((Lc << 1) & ~kRow0) | ((window(mP, c0 - W - 1, nthr) >> 3) & kRow0 & cm.hu & cm.xl);
  n.UR = ((Rc << 1) & ~kRow0) | ((window(mP, c0 - W + 1, nthr) >> 3) & kRow0 & cm.hu & cm.xr);
  n.DL = ((Lc >> 1) & ~kRow3) | ((window(mQ, c0 + W - 1, nthr) << 3) & kRow3 & cm.hd & cm.xl);
  n.DR = ((Rc >> 1) & ~kRow3) | ((window(mQ, c0 + W + 1, nthr) << 3) & kRow3 & cm.hd & cm.xr);
  return n;
}

T1_HD u64 any_of(const Nb &n) { return n.L | n.R | n.U | n.D | n.UL | n.UR | n.DL | n.DR; }

// signs of the horizontal and vertical neighbours (only read where the neighbour is significant)
struct Sg {
  u64 L, R, U, D;
};

T1_HD Sg sign_neighbours(u64 G, const u64 *sg, int t, int nthr, int W) {
  const int c0 = 16 * t;
  Sg s;
  s.L = (G << 4) | (t > 0 ? (sg[t - 1] >> 60) : 0ull);
  s.R = (G >> 4) | (t + 1 < nthr ? (sg[t + 1] << 60) : 0ull);
  s.U = ((G << 1) & ~kRow0) | ((window(sg, c0 - W, nthr) >> 3) & kRow0);
  s.D = ((G >> 1) & ~kRow3) | ((window(sg, c0 + W, nthr) << 3) & kRow3);
  return s;
}

T1_HD uint32_t bitat(u64 m, int p) { return (uint32_t)(m >> p) & 1u; }

// significance-propagation / cleanup decision symbol of sample p
T1_HD uint32_t sig_symbol(const Nb &n, int p, uint32_t bit, const uint8_t *sig2ctx) {
  const uint32_t h = bitat(n.L, p) + bitat(n.R, p);
  const uint32_t v = bitat(n.U, p) + bitat(n.D, p);
  const uint32_t d = bitat(n.UL, p) + bitat(n.UR, p) + bitat(n.DL, p) + bitat(n.DR, p);
  return ((dev::kCtxSig + sig2ctx[15 * h + 5 * v + d]) << 1) | bit;
}

// sign symbol of sample p (tier1.c:264-275 context tables)
T1_HD uint32_t sign_symbol(const Nb &n, const Sg &s, u64 G, int p, const uint8_t *sig2xi,
                           const uint8_t *xi2cont) {
  const uint32_t xh = bitat(n.L, p) | (bitat(n.R, p) << 1) | (bitat(s.L, p) << 2) | (bitat(s.R, p) << 3);
  const uint32_t xv = bitat(n.U, p) | (bitat(n.D, p) << 1) | (bitat(s.U, p) << 2) | (bitat(s.D, p) << 3);
  const uint32_t e = xi2cont[(sig2xi[xh] << 2) | sig2xi[xv]];
  return ((e & 0x7Fu) << 1) | (bitat(G, p) ^ (e >> 7));
}

// sum of the 5-bit values (bit planes P[0] = b-1 most significant .. P[4] = b-5) over mask m
T1_HD long long sum5(u64 m, const u64 *P) {
  return 16ll * popc64(m & P[0]) + 8ll * popc64(m & P[1]) + 4ll * popc64(m & P[2]) +
         2ll * popc64(m & P[3]) + popc64(m & P[4]);
}

// distortion decrease of the samples in m becoming significant at this plane: 49152 + 6144 i
// with i the five magnitude bits below the plane (tier1.c:157-165)
T1_HD long long dist_new(u64 m, const u64 *P) {
  return 49152ll * popc64(m) + 6144ll * sum5(m, P);
}

// distortion change of the samples in m refined at this plane: with i the six bits below the
// plane, 49152 - 2048 i for i < 32 and 2048 i - 81920 above (tier1.c:139-155)
T1_HD long long dist_refine(u64 m, const u64 *P) {
  const u64 m1 = m & P[0], m0 = m & ~P[0];
  return 49152ll * popc64(m0) - 2048ll * sum5(m0, P + 1) - 16384ll * popc64(m1) +
         2048ll * sum5(m1, P + 1);
}

// 8x8 bit-matrix transpose: bit 8k + j -> bit 8j + k
T1_HD u64 transpose8(u64 x) {
  u64 s;
  s = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x = x ^ s ^ (s << 7);
  s = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x = x ^ s ^ (s << 14);
  s = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x = x ^ s ^ (s << 28);
  return x;
}

// Block interface the body needs (CUDA block or host threads):
//   int tid; void sync(); int sync_or(int); uint32_t scan(uint32_t v, uint32_t *total)
//   (exclusive, every thread gets the total); uint32_t reduce_max(uint32_t);
//   void add(long long *shared, long long v); unsigned long long reserve(unsigned long long
//   *counter, unsigned long long n) (global atomic add, thread 0 only);
//   void copy16(uint8_t *dst, const uint8_t *src, uint32_t n16) (block-wide 16-byte copy);
//   void or_flag(uint32_t *flags, uint32_t v) (thread 0 only).
// Every return is taken by all threads together.
#pragma nv_exec_check_disable
template <class Blk>
T1_HD void model_codeblock(Blk &blk, ModelShared &sm, uint8_t *stage, const bwc_float *work,
                           const CbDev &cb, const SbDev &sb, const T1EncOut &out, uint32_t c,
                           const uint8_t *tab_sig2ctx, const uint8_t *tab_sig2xi,
                           const uint8_t *tab_xi2cont) {
  const int t = blk.tid;
  const uint32_t W = cb.w, H = cb.h;
  const uint32_t nstripes = (H + 3) >> 2, nfull = H >> 2, rem = H & 3;
  const uint32_t ncols = W * nstripes * cb.d * cb.nt;
  const int nthr = (int)((ncols + 15) >> 4);
  const ColMasks cm = col_masks(t, W, nstripes, nfull, rem, ncols);
  const int Wi = (int)W;
  if (t < 45) sm.sig2ctx[t] = tab_sig2ctx[sb.cls * 45 + t];
  if (t < 16) sm.sig2xi[t] = tab_sig2xi[t];
  if (t < 11) sm.xi2cont[t] = tab_xi2cont[t];

  // ---- quantisation: signs and bit lengths, then the bit planes ------------------------------
  // sample p = 4i + r of this thread: column 16t + i, row r; pair k of columns (2k, 2k + 1)
  const uint64_t sy = cb.sy, sz = cb.sz, st_ = cb.st;
  uint32_t x0 = 0, j0 = 0, sl0 = 0;
  if (t < nthr) {
    const uint32_t c0 = 16u * (uint32_t)t;
    x0 = c0 % W;
    const uint32_t sr = c0 / W;
    j0 = sr % nstripes;
    sl0 = sr / nstripes;
  }
  // quantised samples of column pair k (8 values, sample 4 * (i & 1) + r)
  auto quantise_pair = [&](int k, bwc_raw q[8], u64 *signs) {
    uint32_t x = x0, j = j0, sl = sl0;
    for (int i = 0; i < 2 * k; ++i) {
      if (++x == W) {
        x = 0;
        if (++j == nstripes) {
          j = 0;
          ++sl;
        }
      }
    }
    for (int h = 0; h < 2; ++h) {
      const int i = 2 * k + h;
      for (int r = 0; r < 4; ++r) {
        q[4 * h + r] = 0;
        if (!((cm.valid >> (4 * i + r)) & 1ull)) continue;
        const uint32_t y = 4 * j + (uint32_t)r, z = sl % cb.d, tt = sl / cb.d;
        const uint64_t idx = cb.base + (uint64_t)(cb.x0 + x) + (uint64_t)(cb.y0 + y) * sy +
                             (uint64_t)(cb.z0 + z) * sz + (uint64_t)(cb.t0 + tt) * st_;
        const bwc_raw raw = raw_of(work[idx]);
        if (signs) *signs |= (u64)(raw >> kPrecBit) << (4 * i + r);
        q[4 * h + r] = quantise(float_of(raw & ~kSignMask), sb.qt_eff);
      }
      if (++x == W) {
        x = 0;
        if (++j == nstripes) {
          j = 0;
          ++sl;
        }
      }
    }
  };
  u64 G = 0;
  uint32_t kb = 0;
  if (t < nthr) {
    for (int k = 0; k < 8; ++k) {
      bwc_raw q[8];
      quantise_pair(k, q, &G);
      for (int s = 0; s < 8; ++s) {
        const uint32_t bl = (uint32_t)bitlen_raw(q[s]);
        kb = kb > bl ? kb : bl;
      }
    }
  }
  const int K = (int)blk.reduce_max(kb);
  if (K == 0) {
    if (t == 0) {
      out.K[c] = 0;
      out.Z[c] = 0;
      out.S[(uint64_t)c * (kMaxPasses + 1)] = 0xFFFF;
    }
    return;
  }
  uint8_t *planes = out.planes + cb.scratch_off;
  const uint64_t pstride = 8ull * (uint64_t)nthr;   // bytes per plane
  if (t < nthr) {
    for (int k = 0; k < 8; ++k) {
      bwc_raw q[8];
      quantise_pair(k, q, nullptr);
      for (int g = 0; 8 * g < K; ++g) {
        u64 m = 0;
        for (int s = 0; s < 8; ++s) m |= (u64)((q[s] >> (8 * g)) & 0xFF) << (8 * s);
        m = transpose8(m);
        for (int jb = 0; jb < 8 && 8 * g + jb < K; ++jb)
          planes[(uint64_t)(8 * g + jb) * pstride + 8ull * t + k] = (uint8_t)(m >> (8 * jb));
      }
    }
  }
  // the codeblock's stream, sized for the worst case at K planes
  if (t == 0) {
    const unsigned long long need = stream_bound(ncols, (uint32_t)K);
    const unsigned long long base = blk.reserve(out.sym_used, need);
    sm.ok = (base + need <= out.sym_cap) ? 1u : 0u;
    sm.base = base;
    if (!sm.ok) blk.or_flag(out.flags + c, 8u);
    out.K[c] = (uint8_t)K;
    out.Z[c] = (uint8_t)(3 * K - 2);
  }
  sm.sgn[t] = G;
  sm.sig[t] = 0;
  if (t < 2) sm.dsum[t] = 0;
  blk.sync();   // planes, signs, stream base visible
  if (!sm.ok) return;
  uint8_t *stream = out.symbols + sm.base;
  uint64_t pos = 0;   // the next pass's chunk, relative to the stream base
  uint32_t *pcount = out.pass_count + (uint64_t)c * kMaxPasses;
  uint64_t *poff = out.pass_off + (uint64_t)c * kMaxPasses;
  int64_t *dmse = out.dmse + (uint64_t)c * kMaxPasses;
  int pass = 0;
  unsigned long long decisions = 0;   // the codeblock's coded decisions (block-uniform)

  auto load_plane = [&](int b) -> u64 {
    if (b < 0 || t >= nthr) return 0ull;
    u64 v;
    const uint8_t *src = planes + (uint64_t)b * pstride + 8ull * t;
#ifdef __CUDA_ARCH__
    v = *reinterpret_cast<const u64 *>(src);
#else
    std::memcpy(&v, src, 8);
#endif
    return v;
  };
  // B = plane b, P[0..5] = planes b-1 .. b-6
  u64 B = load_plane(K - 1);
  u64 P[6];
  for (int i = 0; i < 6; ++i) P[i] = load_plane(K - 2 - i);

  u64 SIG = 0, PI = 0, DEL = 0;
  const bool erres = sb.erres != 0;

  // one pass's output: thread's count n and distortion d, then emit(o) writes its symbols from
  // stage[o]; the block places them, copies the staging area to the pass's chunk and records
  // the pass
  auto finish_pass = [&](uint32_t n, long long d, auto emit) {
    long long *ds = &sm.dsum[pass & 1];
    blk.add(ds, d);
    uint32_t total;
    const uint32_t off = blk.scan(n, &total);   // syncs: sums and counts complete
    // the other sum was last read before this scan and is next added to after the sync below
    if (t == 1) sm.dsum[(pass + 1) & 1] = 0;
    emit(stage + off);
    blk.sync();   // staging complete
    const uint32_t n16 = (total + 15) >> 4;
    blk.copy16(stream + pos, stage, n16);
    if (t == 0) {
      pcount[pass] = total;
      poff[pass] = sm.base + pos;
      dmse[pass] = *ds;
    }
    pos += 16ull * n16;
    decisions += total;
    ++pass;
  };

  for (int b = K - 1; b >= 0; --b) {
    if (b != K - 1) {
      // ---- significance propagation ---------------------------------------------------------
      const u64 cand = ~SIG & cm.valid;
      const u64 cb1 = cand & B;
      u64 *fa = sm.fin[0], *fb = sm.fin[1];
      fa[t] = SIG;
      // neighbours scanned later show their state before the pass: right column, rows below,
      // stripe below
      const u64 Rc = ((SIG >> 4) | (t + 1 < nthr ? (sm.sig[t + 1] << 60) : 0ull)) & cm.xr;
      const u64 pre = Rc | ((Rc << 1) & ~kRow0) | ((Rc >> 1) & ~kRow3) | ((SIG >> 1) & ~kRow3) |
                      ((window(sm.sig, 16 * t + Wi, nthr) << 3) & kRow3 & cm.hd) |
                      ((window(sm.sig, 16 * t + Wi - 1, nthr) << 3) & kRow3 & cm.hd & cm.xl) |
                      ((window(sm.sig, 16 * t + Wi + 1, nthr) << 3) & kRow3 & cm.hd & cm.xr);
      u64 F = SIG;
      if (blk.sync_or(cb1 != 0ull)) {
        for (int it = 0;; ++it) {
          u64 Fn = F;
          if (cb1) {
            const u64 Lb = (t > 0) ? (fa[t - 1] >> 60) : 0ull;
            const u64 ext = ((window(fa, 16 * t - Wi, nthr) >> 3) & kRow0 & cm.hu) |
                            ((window(fa, 16 * t - Wi - 1, nthr) >> 3) & kRow0 & cm.hu & cm.xl) |
                            ((window(fa, 16 * t - Wi + 1, nthr) >> 3) & kRow0 & cm.hu & cm.xr);
            for (int guard = 0; guard < 65; ++guard) {
              const u64 Lc = ((Fn << 4) | Lb) & cm.xl;
              const u64 post = ((Fn << 1) & ~kRow0) | Lc | ((Lc << 1) & ~kRow0) |
                               ((Lc >> 1) & ~kRow3) | ext;
              const u64 f2 = SIG | (cb1 & (pre | post));
              if (f2 == Fn) break;
              Fn = f2;
            }
          }
          fb[t] = Fn;
          const int changed = blk.sync_or(Fn != F);
          F = Fn;
          u64 *tmp = fa;
          fa = fb;
          fb = tmp;
          if (!changed) break;
          if (it > 64 * kModelBlock) {   // cannot happen: every round adds a significant sample
            if (t == 0) blk.or_flag(out.flags + c, 16u);
            break;
          }
        }
      }
      // fa holds every thread's final state after the pass
      const Nb n = neighbours(F, SIG, fa, sm.sig, t, nthr, Wi, cm);
      const u64 V = cand & any_of(n);
      const u64 NEW = V & B;
      const uint32_t cnt = (uint32_t)(popc64(V) + popc64(NEW));
      Sg sg{0, 0, 0, 0};
      if (NEW) sg = sign_neighbours(G, sm.sgn, t, nthr, Wi);
      finish_pass(cnt, dist_new(NEW, P), [&](uint8_t *o) {
        u64 m = V;
        while (m) {
          const int p = ctz64(m);
          m &= m - 1;
          const uint32_t bit = bitat(B, p);
          *o++ = (uint8_t)sig_symbol(n, p, bit, sm.sig2ctx);
          if (bit) *o++ = (uint8_t)sign_symbol(n, sg, G, p, sm.sig2xi, sm.xi2cont);
        }
      });
      PI = V;
      SIG = F;
      sm.sig[t] = SIG;   // every read of the state before the pass happened before the scan
      blk.sync();

      // ---- magnitude refinement -------------------------------------------------------------
      const u64 M = SIG & ~PI & cm.valid;
      const u64 FIRST = M & ~DEL;
      u64 ANY = 0;
      if (FIRST) ANY = any_of(neighbours(SIG, SIG, sm.sig, sm.sig, t, nthr, Wi, cm));
      finish_pass((uint32_t)popc64(M), dist_refine(M, P), [&](uint8_t *o) {
        u64 m = M;
        if (!FIRST) {
          while (m) {
            const int p = ctz64(m);
            m &= m - 1;
            *o++ = (uint8_t)(((dev::kCtxMag + 2) << 1) | bitat(B, p));
          }
        } else {
          while (m) {
            const int p = ctz64(m);
            m &= m - 1;
            const uint32_t ctx = bitat(DEL, p) ? dev::kCtxMag + 2
                                               : dev::kCtxMag + bitat(ANY, p);
            *o++ = (uint8_t)((ctx << 1) | bitat(B, p));
          }
        }
      });
      DEL |= M;
    }

    // ---- cleanup ----------------------------------------------------------------------------
    {
      const u64 cand = ~SIG & ~PI & cm.valid;
      const u64 FCU = SIG | (cand & B);
      sm.fin[0][t] = FCU;
      blk.sync();
      const Nb n = neighbours(FCU, SIG, sm.fin[0], sm.sig, t, nthr, Wi, cm);
      // run mode: full columns whose samples are all insignificant and unvisited and whose
      // neighbourhood (left column and stripe above after the pass, the rest before it) is
      // empty
      const u64 around = n.L | n.R | n.UL | n.UR | n.DL | n.DR | n.Uext | n.Dext | SIG | PI;
      uint32_t runcols = 0;
      for (int i = 0; i < 16; ++i) {
        const u64 nib = 0xFull << (4 * i);
        if ((cm.full & nib) && !(around & nib)) runcols |= 1u << i;
      }
      // counts: columns outside run mode code every candidate (plus its sign if it becomes
      // significant); a run column codes one run bit, or with a set bit at row r0 the run bit,
      // two position bits, r0's sign and the rows below r0 like any candidate
      u64 runmask = 0;
      for (int i = 0; i < 16; ++i)
        if (runcols & (1u << i)) runmask |= 0xFull << (4 * i);
      const u64 cnr = cand & ~runmask;
      uint32_t cnt = (uint32_t)(popc64(cnr) + popc64(cnr & B));
      for (uint32_t rc = runcols; rc; rc &= rc - 1) {
        const int i = ctz64(rc);
        const uint32_t bn = (uint32_t)(B >> (4 * i)) & 0xFu;
        if (!bn) {
          cnt += 1;
        } else {
          const int r0 = ctz64(bn);
          const uint32_t after = (bn >> (r0 + 1));
          cnt += 4 + (uint32_t)(3 - r0) + (uint32_t)popc64(after);
        }
      }
      if (erres && t == kModelBlock - 1) cnt += 4;
      const u64 NEW = cand & B;
      Sg sg{0, 0, 0, 0};
      if (NEW) sg = sign_neighbours(G, sm.sgn, t, nthr, Wi);
      finish_pass(cnt, dist_new(NEW, P), [&](uint8_t *o) {
        u64 todo = cand | runmask;
        while (todo) {
          const int i = ctz64(todo) >> 2;
          const u64 nib = 0xFull << (4 * i);
          todo &= ~nib;
          const uint32_t bn = (uint32_t)(B >> (4 * i)) & 0xFu;
          int r = 0;
          if (runcols & (1u << i)) {
            if (!bn) {
              *o++ = (uint8_t)(dev::kCtxRun << 1);
              continue;
            }
            const int r0 = ctz64(bn);
            *o++ = (uint8_t)((dev::kCtxRun << 1) | 1);
            *o++ = (uint8_t)((dev::kCtxUni << 1) | (uint32_t)(r0 >> 1));
            *o++ = (uint8_t)((dev::kCtxUni << 1) | (uint32_t)(r0 & 1));
            *o++ = (uint8_t)sign_symbol(n, sg, G, 4 * i + r0, sm.sig2xi, sm.xi2cont);
            r = r0 + 1;
          }
          for (; r < 4; ++r) {
            const int p = 4 * i + r;
            if (!bitat(cand, p)) continue;
            const uint32_t bit = bitat(B, p);
            *o++ = (uint8_t)sig_symbol(n, p, bit, sm.sig2ctx);
            if (bit) *o++ = (uint8_t)sign_symbol(n, sg, G, p, sm.sig2xi, sm.xi2cont);
          }
        }
        if (erres && t == kModelBlock - 1) {
          *o++ = (uint8_t)((dev::kCtxUni << 1) | 1);
          *o++ = (uint8_t)(dev::kCtxUni << 1);
          *o++ = (uint8_t)((dev::kCtxUni << 1) | 1);
          *o++ = (uint8_t)(dev::kCtxUni << 1);
        }
      });
      SIG = FCU;
      PI = 0;
      sm.sig[t] = SIG;
      blk.sync();
    }
    // next plane
    B = P[0];
    for (int i = 0; i < 5; ++i) P[i] = P[i + 1];
    P[5] = load_plane(b - 7);
  }
  if (t == 0) blk.reserve(out.sym_used + 1, decisions);
}

}  // namespace t1
}  // namespace bwcb
