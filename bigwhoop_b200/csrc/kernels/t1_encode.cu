// EBCOT tier-1 encoder: quantisation, bit-plane coding passes, MQ coding, minimal truncation
// lengths and convex-hull rate-distortion slopes -- one codeblock per warp.
//
// Reference: cblkcopy_forward (tier1.c:526-729), the three coding passes (tier1.c:962-1511),
// encode_codeblock (tier1.c:2303-2588), the MQ coder (mq.c:85-127, :328-556, :587-759,
// :1151-1175), slope2log and compute_convex_hull (tier1.c:2100-2267).
//
// Work decomposition.  The reference codes a codeblock sample by sample: slices, stripe rows
// of four samples, columns left to right, samples top to bottom.  Here a warp owns a codeblock
// and processes one stripe row per step with one lane per column (chunks of 32 columns):
//   * magnitude refinement: every context depends on state from before the pass -> lanes
//     form their symbols independently;
//   * cleanup: a sample's significance after the pass does not depend on its neighbours, so the
//     left neighbour's final state is known in closed form;
//   * significance propagation: a sample is coded only next to an already significant sample,
//     and significance spreads left to right within the pass.  Lanes iterate
//     column(left-neighbour estimate) -> shuffle until no estimate changes; starting from the
//     pre-pass state the iterates grow monotonically to the sequential result (lane 0's input
//     is exact, so after i rounds the first i lanes are exact).
// Each lane writes its column's symbols (context, decision) to shared memory, and lane 0 feeds
// them to the MQ coder in scan order.  Coder state is recorded at the end of every pass; after
// termination all lanes compute the minimal truncation lengths, and lane 0 builds the convex
// hull of (length, distortion) and the 16-bit log slopes.
//
// Per-codeblock state lives in shared memory: one 16-bit word per stripe column
// (bits 0-3 significance, 4-7 sign, 8-11 "coded in this significance pass", 12-15 refined).
// Quantised magnitudes are stored as bit planes in global memory, one byte per stripe column
// per plane (the column's four bits in the low nibble, row 0 at bit 3).
#include <cstdio>

#include "device_common.cuh"
#include "t1_tables.cuh"

namespace bwcb {
namespace {

using dev::kCtxMag;
using dev::kCtxRun;
using dev::kCtxSig;
using dev::kCtxUni;

constexpr int kWarpsPerBlock = 4;
constexpr int kSymPerLane = 12;

struct Mq {
  uint32_t A, C, T;
  int32_t t;
  int32_t L;
};

struct CbCtx {
  uint8_t *out;
  uint32_t cap;
  uint32_t *flags;
};

__device__ __forceinline__ void mq_transfer(Mq &e, const CbCtx &cc) {
  if (e.T == 0xFF) {
    if (e.L >= 0) {
      if ((uint32_t)e.L < cc.cap) cc.out[e.L] = (uint8_t)e.T; else *cc.flags |= 1u;
    }
    e.L++;
    e.T = (e.C >> 20) & 0xFF;
    e.C &= 0xFFFFF;
    e.t = 7;
  } else {
    if (e.C & 0x8000000) {
      e.T++;
      e.C &= 0x7FFFFFF;
    }
    if (e.L >= 0) {
      if ((uint32_t)e.L < cc.cap) cc.out[e.L] = (uint8_t)e.T; else *cc.flags |= 1u;
    }
    e.L++;
    if (e.T == 0xFF) {
      e.T = (e.C >> 20) & 0xFF;
      e.C &= 0xFFFFF;
      e.t = 7;
    } else {
      e.T = (e.C >> 19) & 0xFF;
      e.C &= 0x7FFFF;
      e.t = 8;
    }
  }
}

__device__ __forceinline__ void mq_encode(Mq &e, uint8_t *ctx, int k, int s, const CbCtx &cc) {
  const uint32_t ent = dev::c_mq_states[ctx[k]];
  const uint32_t p = ent & 0xFFFF;
  e.A -= p;
  if (s == (int)((ent >> 16) & 1)) {
    if (e.A >= 0x8000) {
      e.C += p;
      return;
    }
    if (e.A < p) e.A = p; else e.C += p;
    ctx[k] = (uint8_t)((ent >> 17) & 0x7F);
  } else {
    if (e.A < p) e.C += p; else e.A = p;
    ctx[k] = (uint8_t)((ent >> 24) & 0x7F);
  }
  do {
    e.A <<= 1;
    e.C <<= 1;
    if (--e.t == 0) mq_transfer(e, cc);
  } while (e.A < 0x8000);
}

__device__ void mq_terminate(Mq &e, const CbCtx &cc) {
  int n = 12 - e.t;
  e.C <<= e.t;
  while (n > 0) {
    mq_transfer(e, cc);
    n -= e.t;
    e.C <<= e.t;
  }
  mq_transfer(e, cc);
}

// Minimal number of bytes that decode a pass correctly, given the coder state at its end and the
// bytes emitted later (mq.c:587-675; the single-precision build uses 32-bit split arithmetic).
// Bytes at or beyond `cap` read as zero (the reference's buffer is zero-filled past its data);
// a scan that has not settled after 64 bytes sets *bad (it settles within a few bytes).
__device__ int64_t truncation_length(uint32_t A, uint32_t C, int32_t t, uint32_t T, int64_t L,
                                     const uint8_t *b0, uint32_t cap, uint32_t *bad) {
  struct Bytes {
    const uint8_t *p;
    int64_t cap;
    __device__ __forceinline__ uint32_t operator[](int64_t i) const {
      return (i >= 0 && i < cap) ? p[i] : 0u;
    }
  } b{b0, (int64_t)cap};
  int guard = 0;
#ifdef BWC_SINGLE_PRECISION
  int32_t CrFrac = (int32_t)((uint32_t)C << t);
  int32_t CArFrac = (int32_t)((uint32_t)A << t) + CrFrac;
  int32_t CrDec = (int32_t)T, CArDec = (int32_t)T;
  CrDec += 0x01 & (CrFrac >> 27);
  CArDec += 0x01 & (CArFrac >> 27);
  CrFrac &= 0x7FFFFFF;
  CArFrac &= 0x7FFFFFF;
  int s = 8;
  while ((CrDec > 0xff) || (CArDec <= 0xff)) {
    if (++guard > 64) {
      *bad = 1;
      break;
    }
    const int32_t buff = (L >= 0) ? (int32_t)b[L] : 0;
    L++;
    CrDec -= buff << (8 - s);
    CArDec -= buff << (8 - s);
    CrDec = (int32_t)((uint32_t)CrDec << s);
    CArDec = (int32_t)((uint32_t)CArDec << s);
    CrDec += CrFrac >> (27 - s);
    CArDec += CArFrac >> (27 - s);
    CrFrac = (int32_t)((uint32_t)CrFrac << s);
    CArFrac = (int32_t)((uint32_t)CArFrac << s);
    CrFrac &= 0x7FFFFFF;
    CArFrac &= 0x7FFFFFF;
    s = (buff == 0xFF) ? 7 : 8;
  }
#else
  int64_t Cr = ((int64_t)T << 27) + ((int64_t)C << t);
  int64_t CAr = ((int64_t)A << t) + Cr;
  int s = 8;
  while (((Cr >> 27) > 0xff) || ((CAr >> 27) <= 0xff)) {
    if (++guard > 64) {
      *bad = 1;
      break;
    }
    const int64_t buff = (L >= 0) ? (int64_t)b[L] : 0;
    L++;
    Cr -= buff << (35 - s);
    CAr -= buff << (35 - s);
    Cr = (int64_t)((uint64_t)Cr << s);
    CAr = (int64_t)((uint64_t)CAr << s);
    s = (buff == 0xFF) ? 7 : 8;
  }
#endif
  if (L > 0 && b[L - 1] == 0xFF) L--;
  while (L > 1 && b[L - 2] == 0xFF && b[L - 1] == 0x7F) L -= 2;
  return L;
}

__device__ uint16_t slope2log(double lambda) {
  const uint64_t raw = (uint64_t)__double_as_longlong(lambda);
  const uint64_t exponent = ((raw & 0x7FF0000000000000ull) >> 44) - 0x41F00ull;
  const uint64_t mantissa = (raw & 0x000FFFFFFFFFFFFFull) >> 44;
  const uint64_t r = (exponent + dev::c_frac2log[mantissa]) + 0x10000ull;
  if (r > 0xFFFF) return 0xFFFF;
  if (r < 2) return 2;
  return (uint16_t)r;
}

// Neighbourhood of one stripe column: significance/sign bytes (sigma | xi << 4).
struct Nbr {
  uint32_t L, R, U, UL, UR, D, DL, DR;
};

__device__ __forceinline__ uint32_t bit(uint32_t v, int i) { return (i >= 0 && i < 4) ? (v >> i) & 1u : 0u; }

// 6-bit window of magnitude bits below plane b for row l: bit(b-1) << 5 | ... | bit(b-6)
struct Window {
  uint32_t p[6];
  __device__ __forceinline__ uint32_t w6(int l) const {
    return (((p[0] >> l) & 1) << 5) | (((p[1] >> l) & 1) << 4) | (((p[2] >> l) & 1) << 3) |
           (((p[3] >> l) & 1) << 2) | (((p[4] >> l) & 1) << 1) | ((p[5] >> l) & 1);
  }
};

__device__ __forceinline__ void load_window(Window &w, const uint8_t *planes, uint32_t ncols,
                                           uint32_t col, int b) {
#pragma unroll
  for (int i = 0; i < 6; ++i) w.p[i] = (b - 1 - i >= 0) ? planes[(uint64_t)(b - 1 - i) * ncols + col] : 0u;
}

__device__ __forceinline__ uint32_t sig_index(uint32_t sig, const Nbr &n, int l, bool full) {
  const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF;
  uint32_t kh = bit(Ls, l) + bit(Rs, l);
  uint32_t kv = bit(sig, l + 1) + bit(sig, l - 1);
  uint32_t kd = bit(Ls, l + 1) + bit(Ls, l - 1) + bit(Rs, l + 1) + bit(Rs, l - 1);
  if (l == 3) {
    kv += n.U & 1;
    kd += (n.UL & 1) + (n.UR & 1);
  } else if (l == 0 && full) {
    kv += (n.D >> 3) & 1;
    kd += ((n.DL >> 3) & 1) + ((n.DR >> 3) & 1);
  }
  return 15 * kh + 5 * kv + kd;
}

__device__ __forceinline__ uint32_t sign_symbol(uint32_t sig, uint32_t xi, const Nbr &n, int l,
                                                bool full, uint32_t *ctx_out) {
  const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF, Lx = n.L >> 4, Rx = n.R >> 4;
  const uint32_t xh = bit(Ls, l) | (bit(Rs, l) << 1) | (bit(Lx, l) << 2) | (bit(Rx, l) << 3);
  uint32_t xv = bit(sig, l + 1) | (bit(sig, l - 1) << 1) | (bit(xi, l + 1) << 2) | (bit(xi, l - 1) << 3);
  if (l == 3) {
    xv |= (n.U & 1) | (((n.U >> 4) & 1) << 2);
  } else if (l == 0 && full) {
    xv |= (((n.D >> 3) & 1) << 1) | (((n.D >> 7) & 1) << 3);
  }
  const uint32_t e = dev::c_xi2cont[(dev::c_sig2xi[xh] << 2) | dev::c_sig2xi[xv]];
  *ctx_out = e & 0x7F;
  return bit(xi, l) ^ (e >> 7);
}

struct Emit {
  uint8_t *sym;
  int n;
  __device__ __forceinline__ void put(uint32_t ctx, uint32_t b) { sym[n++] = (uint8_t)((ctx << 1) | b); }
};

// significance propagation of one column; kEmit == false only computes the final significance
template <bool kEmit>
__device__ __forceinline__ uint32_t sp_column(uint32_t st, uint32_t bits, const Nbr &n, int lmin,
                                              bool full, uint32_t cls, Emit *em, int64_t *mse,
                                              const uint8_t *planes, uint32_t ncols, uint32_t col,
                                              int b, uint32_t *st_out) {
  uint32_t sig = st & 0xF, xi = (st >> 4) & 0xF, pi = (st >> 8) & 0xF;
  const uint32_t vmask = (0xFu >> lmin) << lmin;
  if (((sig ^ 0xF) & vmask) == 0) {
    if (kEmit) *st_out = (st & 0xF0FFu);
    return sig;
  }
  Window w;
  bool wl = false;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (!(sig & m)) {
      const uint32_t ks = sig_index(sig, n, l, full);
      if (ks) {
        const uint32_t bv = (bits >> l) & 1;
        if (kEmit) em->put(kCtxSig + dev::c_sig2ctx[cls][ks], bv);
        if (bv) {
          if (kEmit) {
            uint32_t sctx;
            const uint32_t sb = sign_symbol(sig, xi, n, l, full, &sctx);
            em->put(sctx, sb);
            if (!wl) {
              load_window(w, planes, ncols, col, b);
              wl = true;
            }
            *mse += dev::dist_ts(w.w6(l) >> 1);
          }
          sig |= m;
        }
        pi |= m;
      }
    } else {
      pi &= ~m;
    }
  }
  if (kEmit) *st_out = (st & 0xF000u) | (pi << 8) | (xi << 4) | sig;
  return sig;
}

__device__ __forceinline__ void mr_column(uint32_t st, uint32_t bits, const Nbr &n, int lmin,
                                          bool full, Emit *em, int64_t *mse,
                                          const uint8_t *planes, uint32_t ncols, uint32_t col,
                                          int b, uint32_t *st_out) {
  const uint32_t sig = st & 0xF, pi = (st >> 8) & 0xF;
  uint32_t delta = (st >> 12) & 0xF;
  const uint32_t vmask = (0xFu >> lmin) << lmin;
  const uint32_t todo = sig & ~pi & vmask;
  if (!todo) {
    *st_out = st;
    return;
  }
  Window w;
  load_window(w, planes, ncols, col, b);
  const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (todo & m) {
      uint32_t ctx = kCtxMag;
      if (delta & m) {
        ctx += 2;
      } else {
        uint32_t any = bit(sig, l + 1) | bit(sig, l - 1) | bit(Ls, l) | bit(Rs, l) | bit(Ls, l + 1) |
                       bit(Ls, l - 1) | bit(Rs, l + 1) | bit(Rs, l - 1);
        if (l == 3) any |= (n.U | n.UL | n.UR) & 1;
        if (l == 0 && full) any |= ((n.D | n.DL | n.DR) >> 3) & 1;
        ctx += any ? 1 : 0;
      }
      em->put(ctx, (bits >> l) & 1);
      *mse += dev::dist_tm(w.w6(l));
      delta |= m;
    }
  }
  *st_out = (st & 0x0FFFu) | (delta << 12);
}

__device__ __forceinline__ void cu_column(uint32_t st, uint32_t bits, const Nbr &n, int lmin,
                                          bool full, uint32_t cls, Emit *em, int64_t *mse,
                                          const uint8_t *planes, uint32_t ncols, uint32_t col,
                                          int b, uint32_t *st_out) {
  uint32_t sig = st & 0xF;
  const uint32_t xi = (st >> 4) & 0xF, pi = (st >> 8) & 0xF;
  int r = -1;
  if (full) {
    const uint32_t around = ((n.D | n.DL | n.DR) & 0x8) | ((n.U | n.UL | n.UR) & 0x1) |
                            (n.L & 0xF) | (n.R & 0xF) | sig;
    if (!around) {
      if (bits) {
        r = __clz(bits) - 28;
        em->put(kCtxRun, 1);
        em->put(kCtxUni, (uint32_t)r >> 1);
        em->put(kCtxUni, (uint32_t)r & 1);
      } else {
        r = 4;
        em->put(kCtxRun, 0);
      }
    }
  }
  Window w;
  bool wl = false;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (!(sig & m) && !(pi & m)) {
      if (r >= 0) {
        r--;
      } else {
        const uint32_t ks = sig_index(sig, n, l, full);
        em->put(kCtxSig + dev::c_sig2ctx[cls][ks], (bits >> l) & 1);
      }
      if (bits & m) {
        uint32_t sctx;
        const uint32_t sb = sign_symbol(sig, xi, n, l, full, &sctx);
        em->put(sctx, sb);
        if (!wl) {
          load_window(w, planes, ncols, col, b);
          wl = true;
        }
        *mse += dev::dist_ts(w.w6(l) >> 1);
        sig |= m;
      }
    }
  }
  *st_out = (st & 0xFFF0u) | sig;
}

__device__ __forceinline__ int64_t warp_sum64(int64_t v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct WarpSmem {
  uint8_t ctx[32];
  uint8_t cnt[32];
  uint8_t sym[32 * kSymPerLane];
};

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    t1_encode_kernel(const bwc_float *__restrict__ work, FieldDims dims,
                     const CbDev *__restrict__ cbs, uint32_t ncb, const SbDev *__restrict__ sbs,
                     uint32_t erres, T1EncOut out, uint32_t state_cap, uint16_t *gstate,
                     uint32_t *work_counter) {
  extern __shared__ unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WarpSmem *ws = reinterpret_cast<WarpSmem *>(smem_raw) + wib;
  uint16_t *sstate = reinterpret_cast<uint16_t *>(smem_raw + sizeof(WarpSmem) * kWarpsPerBlock) +
                     (size_t)wib * state_cap;

  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(work_counter, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= ncb) break;
    const CbDev cb = cbs[c];
    const SbDev sb = sbs[cb.sb];
    const uint32_t W = cb.w, H = cb.h, nslices = cb.d * cb.nt;
    const uint32_t nstripes = (H + 3) >> 2, nfull = H >> 2, rem = H & 3;
    const uint32_t ncols = W * nstripes * nslices;
    uint16_t *state = (ncols <= state_cap) ? sstate
                                           : gstate + (cb.scratch_off / sizeof(uint16_t));
    uint8_t *planes = out.planes + cb.scratch_off;
    if (ncols > state_cap) planes += (uint64_t)ncols * sizeof(uint16_t);

    // ---- quantise: K, sign bits, magnitude bit planes ----------------------------------------
    const uint64_t sx = 1, sy = dims.width, sz = dims.width * dims.height,
                   st_ = dims.width * dims.height * dims.depth;
    auto sample_index = [&](uint32_t col, int row, bool *valid) -> uint64_t {
      const uint32_t x = col % W, sr = col / W;
      const uint32_t j = sr % nstripes, sl = sr / nstripes;
      const uint32_t y = 4 * j + row;
      *valid = y < H;
      const uint32_t z = sl % cb.d, t = sl / cb.d;
      return (cb.x0 + x) * sx + (uint64_t)(cb.y0 + y) * sy + (uint64_t)(cb.z0 + z) * sz +
             (uint64_t)(cb.t0 + t) * st_;
    };
    uint32_t kmax = 0;
    for (uint32_t col = lane; col < ncols; col += 32) {
      uint32_t xi = 0;
      for (int row = 0; row < 4; ++row) {
        bool v;
        const uint64_t idx = sample_index(col, row, &v);
        if (!v) continue;
        const bwc_raw raw = dev::as_raw(work[idx]);
        const bwc_raw q = dev::to_raw_rz(dev::fdiv(dev::as_float(raw & ~kSignMask), sb.qt_eff));
        xi |= (uint32_t)(raw >> kPrecBit) << (3 - row);
        const uint32_t bl = (kPrecBit + 1) - (uint32_t)(sizeof(bwc_raw) == 8 ? __clzll((long long)q) : __clz((int)q));
        kmax = max(kmax, q ? bl : 0u);
      }
      state[col] = (uint16_t)(xi << 4);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    const int K = (int)kmax;
    if (K == 0) {
      if (lane == 0) {
        out.K[c] = 0;
        out.Z[c] = 0;
        out.S[(uint64_t)c * (kMaxPasses + 1)] = 0xFFFF;
      }
      continue;
    }
    for (uint32_t col = lane; col < ncols; col += 32) {
      bwc_raw q4[4];
      for (int row = 0; row < 4; ++row) {
        bool v;
        const uint64_t idx = sample_index(col, row, &v);
        q4[row] = 0;
        if (!v) continue;
        const bwc_raw raw = dev::as_raw(work[idx]);
        q4[row] = dev::to_raw_rz(dev::fdiv(dev::as_float(raw & ~kSignMask), sb.qt_eff));
      }
      for (int b = 0; b < K; ++b) {
        const uint32_t nib = (uint32_t)(((q4[0] >> b) & 1) << 3) | (uint32_t)(((q4[1] >> b) & 1) << 2) |
                             (uint32_t)(((q4[2] >> b) & 1) << 1) | (uint32_t)((q4[3] >> b) & 1);
        planes[(uint64_t)b * ncols + col] = (uint8_t)nib;
      }
    }
    if (lane < dev::kCtxTotal) ws->ctx[lane] = dev::mq_initial_state(lane);
    __syncwarp();

    // ---- coding passes -------------------------------------------------------------------------
    Mq e{0x8000u, 0u, 0u, 12, -1};
    uint32_t flags = 0;
    const CbCtx cc{out.bytes + cb.out_off, cb.out_cap, &flags};
    uint64_t *snaps = out.snaps + (uint64_t)c * kMaxPasses * 2;
    int64_t *dmse = out.dmse + (uint64_t)c * kMaxPasses;
    int pass = 0;
    for (int b = K - 1; b >= 0; --b) {
      const uint8_t *plane = planes + (uint64_t)b * ncols;
      for (int kind = (b == K - 1) ? 2 : 0; kind < 3; ++kind) {
        int64_t mse = 0;
        for (uint32_t sr = 0; sr < nstripes * nslices; ++sr) {
          const uint32_t j = sr % nstripes;
          const bool full = j < nfull;
          const int lmin = full ? 0 : 4 - (int)rem;
          for (uint32_t x0 = 0; x0 < W; x0 += 32) {
            const uint32_t x = x0 + lane;
            const bool valid = x < W;
            const uint32_t col = sr * W + x;
            Nbr nb{0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t st = 0, bits = 0;
            if (valid) {
              st = state[col];
              bits = plane[col];
              if (x > 0) nb.L = state[col - 1] & 0xFF;
              if (x + 1 < W) nb.R = state[col + 1] & 0xFF;
              if (j > 0) {
                nb.U = state[col - W] & 0xFF;
                if (x > 0) nb.UL = state[col - W - 1] & 0xFF;
                if (x + 1 < W) nb.UR = state[col - W + 1] & 0xFF;
              }
              if (j + 1 < nstripes) {
                nb.D = state[col + W] & 0xFF;
                if (x > 0) nb.DL = state[col + W - 1] & 0xFF;
                if (x + 1 < W) nb.DR = state[col + W + 1] & 0xFF;
              }
            }
            __syncwarp();
            Emit em{ws->sym + lane * kSymPerLane, 0};
            uint32_t nst = st;
            if (kind == 0) {
              // significance propagation: fixed point over the left neighbour's final state
              uint32_t Lsig = nb.L & 0xF;
              for (int it = 0; it < 33; ++it) {
                Nbr t = nb;
                t.L = (nb.L & 0xF0) | Lsig;
                const uint32_t mine = valid ? sp_column<false>(st, bits, t, lmin, full, sb.cls,
                                                                nullptr, nullptr, nullptr, 0, 0, 0,
                                                                nullptr)
                                            : 0u;
                uint32_t left = __shfl_up_sync(0xffffffffu, mine, 1);
                if (lane == 0 || x == 0) left = Lsig;
                const bool changed = __any_sync(0xffffffffu, left != Lsig);
                Lsig = left;
                if (!changed) break;
              }
              nb.L = (nb.L & 0xF0) | Lsig;
              if (valid)
                sp_column<true>(st, bits, nb, lmin, full, sb.cls, &em, &mse, planes, ncols, col, b,
                                &nst);
            } else if (kind == 1) {
              if (valid) mr_column(st, bits, nb, lmin, full, &em, &mse, planes, ncols, col, b, &nst);
            } else {
              // cleanup: the left column ends the pass with sig | (bits & ~pi) on valid rows
              const uint32_t vmask = (0xFu >> lmin) << lmin;
              const uint32_t fin = (st & 0xF) | (bits & ~(st >> 8) & vmask);
              uint32_t left = __shfl_up_sync(0xffffffffu, fin & 0xF, 1);
              if (lane != 0 && x != 0) nb.L = (nb.L & 0xF0) | left;
              if (valid) cu_column(st, bits, nb, lmin, full, sb.cls, &em, &mse, planes, ncols, col, b, &nst);
            }
            ws->cnt[lane] = (uint8_t)em.n;
            if (valid) state[col] = (uint16_t)nst;
            __syncwarp();
            if (lane == 0) {
              for (int ln = 0; ln < 32; ++ln) {
                const int cntl = ws->cnt[ln];
                const uint8_t *sp = ws->sym + ln * kSymPerLane;
                for (int i = 0; i < cntl; ++i) mq_encode(e, ws->ctx, sp[i] >> 1, sp[i] & 1, cc);
              }
            }
            __syncwarp();
          }
        }
        if (kind == 2 && erres && lane == 0) {
          mq_encode(e, ws->ctx, kCtxUni, 1, cc);
          mq_encode(e, ws->ctx, kCtxUni, 0, cc);
          mq_encode(e, ws->ctx, kCtxUni, 1, cc);
          mq_encode(e, ws->ctx, kCtxUni, 0, cc);
        }
        mse = warp_sum64(mse);
        if (lane == 0) {
          dmse[pass] = mse;
          snaps[2 * pass] = ((uint64_t)e.A << 48) | ((uint64_t)(e.T & 0xFF) << 40) |
                            ((uint64_t)(uint8_t)e.t << 32) | (uint64_t)e.C;
          snaps[2 * pass + 1] = (uint64_t)(int64_t)e.L;
        }
        pass++;
      }
    }
    const int Z = pass;
    if (lane == 0) {
      mq_terminate(e, cc);
      // zero margin after the flushed bytes: truncation-length scans may look past them
      for (int i = 0; i < 16; ++i) {
        const int64_t p = (int64_t)e.L + i;
        if (p >= 0 && (uint64_t)p < cc.cap) cc.out[p] = 0;
      }
    }
    __syncwarp();
    // ---- truncation lengths ------------------------------------------------------------------
    uint32_t *Lout = out.L + (uint64_t)c * kMaxPasses;
    uint32_t scan_bad = 0;
    for (int j = lane; j < Z; j += 32) {
      const uint64_t s0 = snaps[2 * j];
      const int64_t Ls = (int64_t)snaps[2 * j + 1];
      const uint32_t A = (uint32_t)(s0 >> 48), T = (uint32_t)((s0 >> 40) & 0xFF);
      const int32_t t = (int32_t)(int8_t)((s0 >> 32) & 0xFF);
      const uint32_t C = (uint32_t)s0;
      Lout[j] = (uint32_t)truncation_length(A, C, t, T, Ls, cc.out, cc.cap, &scan_bad);
    }
    if (__any_sync(0xffffffffu, scan_bad)) flags |= 4u;
    __syncwarp();
    // ---- convex hull and log slopes (lane 0) --------------------------------------------------
    if (lane == 0) {
      // scratch reuse: pass distortions overwrite dmse, the slopes and the hull stack the
      // (already consumed) coder snapshots
      double *mse_d = reinterpret_cast<double *>(dmse);
      double *lambda = reinterpret_cast<double *>(snaps);
      uint8_t *hull = reinterpret_cast<uint8_t *>(snaps + kMaxPasses + 1);
      double scale = sb.gain_step2;
      scale = dev::fmul(scale, ldexp(1.0, 2 * K));
      scale = dev::fdiv(scale, 65536.0);
      {
        int j = 0;
        for (int b = K - 1; b >= 0; --b) {
          for (int kind = (b == K - 1) ? 2 : 0; kind < 3; ++kind, ++j)
            mse_d[j] = dev::fmul(__ll2double_rn(dmse[j]), scale);
          scale = dev::fmul(scale, 0.25);
        }
      }
      for (int i = 0; i <= Z; ++i) lambda[i] = 0.0;
      for (int i = 0; i < Z; ++i) hull[i] = 0;
      lambda[0] = 18446744073709551616.0;
      int h = 0, hlast = 0;
      for (int i = 0; i < Z; ++i) {
        double dD = 0.0;
        for (int q = hlast; q <= i; ++q) dD = dev::fadd(dD, mse_d[q]);
        uint64_t dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
        if (dD > 0) {
          while (dD >= dev::fmul(lambda[hlast], __ull2double_rn(dL))) {
            lambda[hlast] = 0;
            if (h == 0) {
              // the reference would read below its hull stack here
              flags |= 2u;
              break;
            }
            h--;
            hlast = hull[h];
            dD = 0.0;
            for (int q = hlast; q <= i; ++q) dD = dev::fadd(dD, mse_d[q]);
            dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
          }
          h++;
          hlast = i + 1;
          hull[h] = (uint8_t)hlast;
          if (dL == 0) {
            lambda[hlast] = (dD < 0) ? -1.0 : (dD == 0 ? 0.0 : 18446744073709551616.0);
          } else {
            lambda[hlast] = dev::fdiv(dD, __ull2double_rn(dL));
          }
        } else {
          lambda[i + 1] = 0;
        }
      }
      uint16_t *S = out.S + (uint64_t)c * (kMaxPasses + 1);
      uint32_t smin = 0xFFFF, smax = 0;
      for (int i = 0; i <= Z; ++i) {
        uint16_t v;
        if (lambda[i] < 0)
          v = 1;
        else if (lambda[i] == 0)
          v = (i == Z) ? 1 : 0;
        else
          v = slope2log(lambda[i]);
        S[i] = v;
        if (v) {
          smin = min(smin, (uint32_t)v);
          smax = max(smax, (uint32_t)v);
        }
      }
      if (Lout[Z - 1] > 0) {
        atomicMin(&out.slopes[0], smin);
        atomicMax(&out.slopes[1], smax);
      }
      out.K[c] = (uint8_t)K;
      out.Z[c] = (uint8_t)Z;
      out.flags[c] = flags;
    }
    __syncwarp();
  }
}

}  // namespace

void launch_t1_encode_ex(const bwc_float *work, const FieldDims &dims, const CbDev *cbs,
                         uint32_t ncb, const SbDev *sbs, uchar erres, const T1EncOut &out,
                         uint32_t state_cap, uint16_t *gstate, uint32_t *work_counter,
                         int grid, cudaStream_t s) {
  const size_t smem = sizeof(WarpSmem) * kWarpsPerBlock +
                      (size_t)state_cap * sizeof(uint16_t) * kWarpsPerBlock;
  cudaFuncSetAttribute(t1_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  t1_encode_kernel<<<grid, kWarpsPerBlock * 32, smem, s>>>(work, dims, cbs, ncb, sbs, erres, out,
                                                            state_cap, gstate, work_counter);
}

}  // namespace bwcb
