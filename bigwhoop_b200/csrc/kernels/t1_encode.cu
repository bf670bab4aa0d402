// EBCOT tier-1 encoder: quantisation, bit-plane coding passes, MQ coding, minimal truncation
// lengths and convex-hull rate-distortion slopes.
//
// Reference: cblkcopy_forward (tier1.c:526-729), the three coding passes (tier1.c:962-1511),
// encode_codeblock (tier1.c:2303-2588), the MQ coder (mq.c:85-127, :328-556, :587-759,
// :1151-1175), slope2log and compute_convex_hull (tier1.c:2100-2267).
//
// Two kernels, run one after the other on the stream.
//
// t1_model_kernel -- one CTA of 256 threads per codeblock, persistent over a device work queue
// (largest codeblocks first).  Quantises the codeblock into bit planes and writes every coding
// pass's decisions (context << 1 | decision, one byte each, in the reference's scan order) into
// the codeblock's symbol stream: passes back to back, each starting on a 16-byte boundary, in one
// region of the shared arena reserved per codeblock for the worst case at its bit-plane count.
// The body is t1_model.cuh (64-bit sample masks per thread; see there).  Codeblocks of more than
// 4096 stripe columns run through t1_model_wide_kernel instead (one stripe column at a time per
// thread, below), which writes the same stream.
//
// t1_mq_kernel -- one lane per codeblock, 1 to 32 codeblocks per warp.  Runs the MQ arithmetic
// coder over the codeblock's stream (t1_mq.cuh: branch-free per decision except byte
// transfers), records the coder state at the end of every pass, terminates, derives the minimal
// truncation length of every pass, builds the convex hull and the 16-bit log slopes
// (t1_common.cuh).
//
// t1_model_wide_kernel's stripe-column state (shared memory, one byte each): lo = significance |
// sign << 4 (read by neighbours), hi = visited-in-significance-pass | refined << 4 (owner only).
// Bit planes: one byte per stripe column per plane, the column's four bits in the low nibble,
// row 0 at bit 3.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "bwc_b200.h"
#include "device_common.cuh"
#include "t1_model.cuh"
#include "t1_mq.cuh"
#include "t1_tables.cuh"

namespace bwcb {
namespace {

using dev::kCtxMag;
using dev::kCtxRun;
using dev::kCtxSig;
using dev::kCtxUni;

constexpr int kModelThreads = 256;
constexpr int kMqThreads = 32;

// ---- geometry and neighbourhood -------------------------------------------------------------

struct Geo {
  uint32_t W, H, nstripes, nfull, rem, nslices, ncols;
};

__device__ __forceinline__ Geo make_geo(const CbDev &cb) {
  Geo g;
  g.W = cb.w;
  g.H = cb.h;
  g.nstripes = (cb.h + 3) >> 2;
  g.nfull = cb.h >> 2;
  g.rem = cb.h & 3;
  g.nslices = cb.d * cb.nt;
  g.ncols = g.W * g.nstripes * g.nslices;
  return g;
}

struct Nbr {
  uint32_t L, R, U, UL, UR, D, DL, DR;   // significance | sign << 4 of the eight neighbours
};

__device__ __forceinline__ uint32_t bit(uint32_t v, int i) {
  return (i >= 0 && i < 4) ? (v >> i) & 1u : 0u;
}

// Neighbourhood of column `col`: left/upper neighbours from `fin` (post-pass significance
// estimates) when given, right/lower from `lo` (pre-pass).  Sign bits always from `lo`.
// stripe-column cursor: col = x + W * (j + nstripes * slice), advanced column by column
__device__ __forceinline__ void advance(uint32_t &x, uint32_t &j, const Geo &g) {
  if (++x == g.W) {
    x = 0;
    if (++j == g.nstripes) j = 0;
  }
}

__device__ __forceinline__ Nbr neighbours(const uint8_t *lo, const uint8_t *fin, const Geo &g,
                                          uint32_t col, uint32_t x, uint32_t j) {
  Nbr n{0, 0, 0, 0, 0, 0, 0, 0};
  auto fl = [&](uint32_t k) -> uint32_t {
    return fin ? ((lo[k] & 0xF0u) | fin[k]) : lo[k];
  };
  if (x > 0) n.L = fl(col - 1);
  if (x + 1 < g.W) n.R = lo[col + 1];
  if (j > 0) {
    n.U = fl(col - g.W);
    if (x > 0) n.UL = fl(col - g.W - 1);
    if (x + 1 < g.W) n.UR = fl(col - g.W + 1);
  }
  if (j + 1 < g.nstripes) {
    n.D = lo[col + g.W];
    if (x > 0) n.DL = lo[col + g.W - 1];
    if (x + 1 < g.W) n.DR = lo[col + g.W + 1];
  }
  return n;
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
  uint32_t xv = bit(sig, l + 1) | (bit(sig, l - 1) << 1) | (bit(xi, l + 1) << 2) |
                (bit(xi, l - 1) << 3);
  if (l == 3) {
    xv |= (n.U & 1) | (((n.U >> 4) & 1) << 2);
  } else if (l == 0 && full) {
    xv |= (((n.D >> 3) & 1) << 1) | (((n.D >> 7) & 1) << 3);
  }
  const uint32_t e = dev::c_xi2cont[(dev::c_sig2xi[xh] << 2) | dev::c_sig2xi[xv]];
  *ctx_out = e & 0x7F;
  return bit(xi, l) ^ (e >> 7);
}

// magnitude bits b-1 .. b-6 of the column's four samples
struct Window {
  uint32_t p[6];
  __device__ __forceinline__ void load(const uint8_t *planes, uint32_t ncols, uint32_t col, int b) {
#pragma unroll
    for (int i = 0; i < 6; ++i)
      p[i] = (b - 1 - i >= 0) ? planes[(uint64_t)(b - 1 - i) * ncols + col] : 0u;
  }
  __device__ __forceinline__ uint32_t w6(int l) const {
    return (((p[0] >> l) & 1) << 5) | (((p[1] >> l) & 1) << 4) | (((p[2] >> l) & 1) << 3) |
           (((p[3] >> l) & 1) << 2) | (((p[4] >> l) & 1) << 1) | ((p[5] >> l) & 1);
  }
};

// symbol sinks: counting, or writing (context << 1 | decision) bytes
struct CountSink {
  uint32_t n = 0;
  __device__ __forceinline__ void put(uint32_t, uint32_t) { ++n; }
};
struct WriteSink {
  uint8_t *p;
  __device__ __forceinline__ void put(uint32_t ctx, uint32_t b) { *p++ = (uint8_t)((ctx << 1) | b); }
};
// symbols held in a thread's shared-memory slice until the pass's offsets are known (a count
// beyond `cap` marks an overflow: the bytes past it are not kept)
struct StageSink {
  uint8_t *p;
  uint32_t cap;
  uint32_t n = 0;
  __device__ __forceinline__ void put(uint32_t ctx, uint32_t b) {
    if (n < cap) p[n] = (uint8_t)((ctx << 1) | b);
    ++n;
  }
};

// ---- per-column pass logic (tier1.c:962-1146, :1177-1301, :1332-1511) -------------------------

// post-pass significance of a column in the significance propagation pass
__device__ __forceinline__ uint32_t sp_outcome(uint32_t sig, uint32_t bits, const Nbr &n,
                                               int lmin, bool full) {
  const uint32_t vmask = (0xFu >> lmin) << lmin;
  if (((sig ^ 0xF) & vmask) == 0) return sig;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (!(sig & m) && (bits & m) && sig_index(sig, n, l, full)) sig |= m;
  }
  return sig;
}

// significance propagation symbols; returns the new "visited" nibble
template <class Sink, bool kDist>
__device__ __forceinline__ uint32_t sp_symbols(uint32_t sig, uint32_t xi, uint32_t pi,
                                               uint32_t bits, const Nbr &n, int lmin, bool full,
                                               uint32_t cls, Sink &sink, int64_t *mse,
                                               const uint8_t *planes, uint32_t ncols,
                                               uint32_t col, int b) {
  const uint32_t vmask = (0xFu >> lmin) << lmin;
  if (((sig ^ 0xF) & vmask) == 0) return 0;
  Window w;
  bool wl = false;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (!(sig & m)) {
      const uint32_t ks = sig_index(sig, n, l, full);
      if (ks) {
        const uint32_t bv = (bits >> l) & 1;
        sink.put(kCtxSig + dev::c_sig2ctx[cls][ks], bv);
        if (bv) {
          uint32_t sctx;
          const uint32_t sb = sign_symbol(sig, xi, n, l, full, &sctx);
          sink.put(sctx, sb);
          if (kDist) {
            if (!wl) {
              w.load(planes, ncols, col, b);
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
  return pi;
}

template <class Sink, bool kDist>
__device__ __forceinline__ uint32_t mr_symbols(uint32_t sig, uint32_t pi, uint32_t delta,
                                               uint32_t bits, const Nbr &n, int lmin, bool full,
                                               Sink &sink, int64_t *mse, const uint8_t *planes,
                                               uint32_t ncols, uint32_t col, int b) {
  const uint32_t vmask = (0xFu >> lmin) << lmin;
  const uint32_t todo = sig & ~pi & vmask;
  if (!todo) return delta;
  Window w;
  if (kDist) w.load(planes, ncols, col, b);
  const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF;
  for (int l = 3; l >= lmin; --l) {
    const uint32_t m = 1u << l;
    if (todo & m) {
      uint32_t ctx = kCtxMag;
      if (delta & m) {
        ctx += 2;
      } else {
        uint32_t any = bit(sig, l + 1) | bit(sig, l - 1) | bit(Ls, l) | bit(Rs, l) |
                       bit(Ls, l + 1) | bit(Ls, l - 1) | bit(Rs, l + 1) | bit(Rs, l - 1);
        if (l == 3) any |= (n.U | n.UL | n.UR) & 1;
        if (l == 0 && full) any |= ((n.D | n.DL | n.DR) >> 3) & 1;
        ctx += any ? 1 : 0;
      }
      sink.put(ctx, (bits >> l) & 1);
      if (kDist) *mse += dev::dist_tm(w.w6(l));
      delta |= m;
    }
  }
  return delta;
}

template <class Sink, bool kDist>
__device__ __forceinline__ void cu_symbols(uint32_t sig, uint32_t xi, uint32_t pi, uint32_t bits,
                                           const Nbr &n, int lmin, bool full, uint32_t cls,
                                           Sink &sink, int64_t *mse, const uint8_t *planes,
                                           uint32_t ncols, uint32_t col, int b) {
  int r = -1;
  if (full) {
    const uint32_t around = ((n.D | n.DL | n.DR) & 0x8) | ((n.U | n.UL | n.UR) & 0x1) |
                            (n.L & 0xF) | (n.R & 0xF) | sig;
    if (!around) {
      if (bits) {
        r = __clz(bits) - 28;
        sink.put(kCtxRun, 1);
        sink.put(kCtxUni, (uint32_t)r >> 1);
        sink.put(kCtxUni, (uint32_t)r & 1);
      } else {
        r = 4;
        sink.put(kCtxRun, 0);
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
        sink.put(kCtxSig + dev::c_sig2ctx[cls][sig_index(sig, n, l, full)], (bits >> l) & 1);
      }
      if (bits & m) {
        uint32_t sctx;
        const uint32_t sb = sign_symbol(sig, xi, n, l, full, &sctx);
        sink.put(sctx, sb);
        if (kDist) {
          if (!wl) {
            w.load(planes, ncols, col, b);
            wl = true;
          }
          *mse += dev::dist_ts(w.w6(l) >> 1);
        }
        sig |= m;
      }
    }
  }
}

// ---- block reductions -------------------------------------------------------------------------

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total,
                                                         uint32_t *wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = (lane < (kModelThreads >> 5)) ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < (kModelThreads >> 5)) wsum[lane] = s;
  }
  __syncthreads();
  const uint32_t base = (w > 0) ? wsum[w - 1] : 0;
  *total = wsum[(kModelThreads >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ int64_t block_sum64(int64_t v, int64_t *wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) wsum[w] = v;
  __syncthreads();
  int64_t s = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (kModelThreads >> 5); ++i) s += wsum[i];
  __syncthreads();
  return s;
}

// ---- kernel 1: quantisation + context modelling ------------------------------------------------

// quantisation and context modelling of codeblock c by the whole CTA (every thread calls it,
// every return is taken by all threads together)
__device__ __forceinline__ void model_codeblock(const bwc_float *__restrict__ work,
                                                const CbDev *__restrict__ cbs,
                                                const SbDev *__restrict__ sbs,
                                                const T1EncOut &out, const uint32_t c,
                                                const uint32_t stage_cap) {
  extern __shared__ uint8_t smem[];
  __shared__ uint32_t s_wsum[kModelThreads / 32];
  __shared__ int64_t s_wsum64[kModelThreads / 32];
  __shared__ uint32_t s_K, s_ok;
  __shared__ uint64_t s_base, s_stream, s_pos, s_decisions;
  const int tid = threadIdx.x;
  const CbDev cb = cbs[c];
  const SbDev sb = sbs[cb.sb];
  const Geo g = make_geo(cb);
  // dynamic shared memory: each thread's symbol staging slice (stage_cap bytes, 0 = none),
  // then the stripe-column states
  uint8_t *stage = smem + (size_t)tid * stage_cap;
  uint8_t *lo = smem + (size_t)kModelThreads * stage_cap, *hi = lo + g.ncols, *fin = lo + 2 * g.ncols;
  uint8_t *planes = out.planes + cb.scratch_off;

  // ---- quantise -------------------------------------------------------------------------------
  const uint64_t sy = cb.sy, sz = cb.sz, st_ = cb.st;
  auto sample = [&](uint32_t col, int row, bool *valid) -> uint64_t {
    const uint32_t x = col % g.W, sr = col / g.W;
    const uint32_t j = sr % g.nstripes, sl = sr / g.nstripes;
    const uint32_t y = 4 * j + row;
    *valid = y < g.H;
    const uint32_t z = sl % cb.d, t = sl / cb.d;
    return cb.base + (uint64_t)(cb.x0 + x) + (uint64_t)(cb.y0 + y) * sy + (uint64_t)(cb.z0 + z) * sz +
           (uint64_t)(cb.t0 + t) * st_;
  };
  auto quant = [&](uint64_t idx, uint32_t *sign) -> bwc_raw {
    const bwc_raw raw = dev::as_raw(work[idx]);
    *sign = (uint32_t)(raw >> kPrecBit);
    return dev::to_raw_rz(dev::fdiv(dev::as_float(raw & ~kSignMask), sb.qt_eff));
  };
  uint32_t kmax = 0;
  for (uint32_t col = tid; col < g.ncols; col += kModelThreads) {
    uint32_t xi = 0;
    for (int row = 0; row < 4; ++row) {
      bool v;
      const uint64_t idx = sample(col, row, &v);
      if (!v) continue;
      uint32_t sgn;
      const bwc_raw q = quant(idx, &sgn);
      xi |= sgn << (3 - row);
      const uint32_t bl = q ? (uint32_t)(8 * sizeof(bwc_raw)) -
                                  (uint32_t)(sizeof(bwc_raw) == 8 ? __clzll((long long)q)
                                                                  : __clz((int)(uint32_t)q))
                            : 0u;
      kmax = max(kmax, bl);
    }
    lo[col] = (uint8_t)(xi << 4);
    hi[col] = 0;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  if (tid == 0) s_K = 0;
  __syncthreads();
  if ((tid & 31) == 0) atomicMax(&s_K, kmax);
  __syncthreads();
  const int K = (int)s_K;
  if (K == 0) {
    if (tid == 0) {
      out.K[c] = 0;
      out.Z[c] = 0;
      out.S[(uint64_t)c * (kMaxPasses + 1)] = 0xFFFF;
    }
    return;
  }
  for (uint32_t col = tid; col < g.ncols; col += kModelThreads) {
    bwc_raw q4[4];
    for (int row = 0; row < 4; ++row) {
      bool v;
      const uint64_t idx = sample(col, row, &v);
      uint32_t sgn;
      q4[row] = v ? quant(idx, &sgn) : (bwc_raw)0;
    }
    for (int b = 0; b < K; ++b) {
      const uint32_t nib = ((uint32_t)((q4[0] >> b) & 1) << 3) | ((uint32_t)((q4[1] >> b) & 1) << 2) |
                           ((uint32_t)((q4[2] >> b) & 1) << 1) | (uint32_t)((q4[3] >> b) & 1);
      planes[(uint64_t)b * g.ncols + col] = (uint8_t)nib;
    }
  }
  if (tid == 0) {
    out.K[c] = (uint8_t)K;
    out.Z[c] = (uint8_t)(3 * K - 2);
    // the codeblock's stream, sized for the worst case at K planes; a full arena marks the
    // codeblock for a retry with a larger one
    const uint64_t need = t1::stream_bound(g.ncols, (uint32_t)K);
    const uint64_t base = atomicAdd(out.sym_used, (unsigned long long)need);
    s_ok = (base + need <= out.sym_cap) ? 1u : 0u;
    s_stream = base;
    s_pos = 0;
    s_decisions = 0;
    if (!s_ok) out.flags[c] |= 8u;
  }
  __syncthreads();   // planes and column states are read across threads from here on
  if (!s_ok) return;
  // Every pass's symbols go to the next 16-byte aligned chunk of the codeblock's stream, placed
  // once the pass's symbol count is known.
  auto reserve = [&](uint32_t total) -> uint8_t * {
    if (tid == 0) {
      s_base = s_stream + s_pos;
      s_pos += ((uint64_t)total + 15) & ~15ull;
      s_decisions += total;
    }
    __syncthreads();
    return out.symbols + s_base;
  };
  // a thread's staged symbols to their place in the pass's chunk; an overflowed slice (not
  // possible: a column yields at most 10 symbols a pass, and the slice holds 10 per column
  // plus 4) marks the codeblock
  auto unstage = [&](const StageSink &ss, uint8_t *dst) {
    const uint32_t n = min(ss.n, ss.cap);
    for (uint32_t i = 0; i < n; ++i) dst[i] = ss.p[i];
    if (ss.n > ss.cap) out.flags[c] |= 16u;
  };

  // ---- coding passes --------------------------------------------------------------------------
  const uint32_t cpt = (g.ncols + kModelThreads - 1) / kModelThreads;
  const uint32_t c0 = min(g.ncols, tid * cpt), c1 = min(g.ncols, c0 + cpt);
  const uint32_t cx0 = c0 % g.W, cj0 = (c0 / g.W) % g.nstripes;   // cursor at c0
  uint32_t *pcount = out.pass_count + (uint64_t)c * kMaxPasses;
  uint64_t *poff = out.pass_off + (uint64_t)c * kMaxPasses;
  int64_t *dmse = out.dmse + (uint64_t)c * kMaxPasses;
  int pass = 0;
  for (int b = K - 1; b >= 0; --b) {
    const uint8_t *plane = planes + (uint64_t)b * g.ncols;
    for (int kind = (b == K - 1) ? 2 : 0; kind < 3; ++kind) {
      int64_t mse = 0;
      if (kind == 0) {
        // significance propagation: fixed point of the post-pass significance
        for (uint32_t col = c0; col < c1; ++col) fin[col] = lo[col] & 0xF;
        __syncthreads();
        // every round that changes anything makes at least one more sample significant, so
        // 4 * ncols + 1 rounds always suffice; the bound only guards against a logic error
        for (uint32_t it = 0; it <= 4 * g.ncols; ++it) {
          int changed = 0;
          for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
            const bool full = j < g.nfull;
            const int lmin = full ? 0 : 4 - (int)g.rem;
            const Nbr n = neighbours(lo, fin, g, col, x, j);
            const uint32_t s = sp_outcome(lo[col] & 0xF, plane[col], n, lmin, full);
            if (s != fin[col]) {
              fin[col] = (uint8_t)s;
              changed = 1;
            }
          }
          if (!__syncthreads_or(changed)) break;
        }
        // the pass's symbols (and, with kDist, its distortion and the visited nibbles)
        auto sp_run = [&](auto &sink, auto dist) {
          constexpr bool kDist = decltype(dist)::value;
          for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
            const bool full = j < g.nfull;
            const int lmin = full ? 0 : 4 - (int)g.rem;
            const Nbr n = neighbours(lo, fin, g, col, x, j);
            const uint32_t pi = sp_symbols<std::remove_reference_t<decltype(sink)>, kDist>(
                lo[col] & 0xF, lo[col] >> 4, hi[col] & 0xF, plane[col], n, lmin, full, sb.cls,
                sink, &mse, planes, g.ncols, col, b);
            if (kDist) hi[col] = (uint8_t)((hi[col] & 0xF0) | pi);
          }
        };
        uint32_t total;
        if (stage_cap) {
          StageSink ss{stage, stage_cap};
          sp_run(ss, std::true_type{});
          const uint32_t off = block_exclusive_scan(ss.n, &total, s_wsum);
          uint8_t *chunk = reserve(total);
          if (!chunk) return;
          unstage(ss, chunk + off);
        } else {
          CountSink cnt;
          sp_run(cnt, std::false_type{});
          const uint32_t off = block_exclusive_scan(cnt.n, &total, s_wsum);
          uint8_t *chunk = reserve(total);
          if (!chunk) return;
          WriteSink ws{chunk + off};
          sp_run(ws, std::true_type{});
        }
        __syncthreads();
        for (uint32_t col = c0; col < c1; ++col) lo[col] = (uint8_t)((lo[col] & 0xF0) | fin[col]);
        if (tid == 0) {
          pcount[pass] = total;
          poff[pass] = s_base;
        }
      } else if (kind == 1) {
        // one refinement symbol per significant sample not visited by this plane's
        // significance pass
        CountSink cnt;
        for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
          const int lmin = (j < g.nfull) ? 0 : 4 - (int)g.rem;
          const uint32_t vmask = (0xFu >> lmin) << lmin;
          cnt.n += __popc((uint32_t)(lo[col] & ~hi[col]) & vmask & 0xFu);
        }
        uint32_t total;
        const uint32_t off = block_exclusive_scan(cnt.n, &total, s_wsum);
        uint8_t *chunk = reserve(total);
        if (!chunk) return;
        WriteSink ws{chunk + off};
        for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
          const bool full = j < g.nfull;
          const int lmin = full ? 0 : 4 - (int)g.rem;
          const uint32_t s = lo[col] & 0xF, p = hi[col] & 0xF, dl0 = hi[col] >> 4;
          if (!(s & ~p)) continue;
          // neighbours only decide the context of a sample's first refinement
          Nbr n{0, 0, 0, 0, 0, 0, 0, 0};
          if (s & ~p & ~dl0) n = neighbours(lo, nullptr, g, col, x, j);
          const uint32_t dl = mr_symbols<WriteSink, true>(s, p, dl0, plane[col], n, lmin,
                                                          full, ws, &mse, planes, g.ncols, col, b);
          hi[col] = (uint8_t)((hi[col] & 0x0F) | (dl << 4));
        }
        if (tid == 0) {
          pcount[pass] = total;
          poff[pass] = s_base;
        }
      } else {
        // cleanup: post-pass significance in closed form
        for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
          const int lmin = (j < g.nfull) ? 0 : 4 - (int)g.rem;
          const uint32_t vmask = (0xFu >> lmin) << lmin;
          fin[col] = (uint8_t)((lo[col] & 0xF) | (plane[col] & ~hi[col] & vmask));
        }
        __syncthreads();
        auto cu_run = [&](auto &sink, auto dist) {
          constexpr bool kDist = decltype(dist)::value;
          for (uint32_t col = c0, x = cx0, j = cj0; col < c1; ++col, advance(x, j, g)) {
            const bool full = j < g.nfull;
            const int lmin = full ? 0 : 4 - (int)g.rem;
            const Nbr n = neighbours(lo, fin, g, col, x, j);
            cu_symbols<std::remove_reference_t<decltype(sink)>, kDist>(
                lo[col] & 0xF, lo[col] >> 4, hi[col] & 0xF, plane[col], n, lmin, full, sb.cls,
                sink, &mse, planes, g.ncols, col, b);
          }
        };
        // with error resilience the last thread appends the segmentation symbol after every
        // bit plane (tier1.c:94-100)
        const bool seg = sb.erres && tid == kModelThreads - 1;
        auto segmark = [&](auto &sink) {
          if (seg) {
            sink.put(kCtxUni, 1);
            sink.put(kCtxUni, 0);
            sink.put(kCtxUni, 1);
            sink.put(kCtxUni, 0);
          }
        };
        uint32_t total;
        if (stage_cap) {
          StageSink ss{stage, stage_cap};
          cu_run(ss, std::true_type{});
          segmark(ss);
          const uint32_t off = block_exclusive_scan(ss.n, &total, s_wsum);
          uint8_t *chunk = reserve(total);
          if (!chunk) return;
          unstage(ss, chunk + off);
        } else {
          CountSink cnt;
          cu_run(cnt, std::false_type{});
          segmark(cnt);
          const uint32_t off = block_exclusive_scan(cnt.n, &total, s_wsum);
          uint8_t *chunk = reserve(total);
          if (!chunk) return;
          WriteSink ws{chunk + off};
          cu_run(ws, std::true_type{});
          segmark(ws);
        }
        __syncthreads();
        for (uint32_t col = c0; col < c1; ++col) lo[col] = (uint8_t)((lo[col] & 0xF0) | fin[col]);
        if (tid == 0) {
          pcount[pass] = total;
          poff[pass] = s_base;
        }
      }
      const int64_t m = block_sum64(mse, s_wsum64);
      if (tid == 0) dmse[pass] = m;
      __syncthreads();
      pass++;
    }
  }
  if (tid == 0) atomicAdd(out.sym_used + 1, (unsigned long long)s_decisions);
}

// Modelling of codeblocks over 4096 stripe columns.  Without a queue, CTA i models codeblock
// order[i] (or i).  With a queue it is persistent: every CTA takes the next position of the
// device work queue (an atomic counter over `order`, largest codeblocks first) until the list is
// exhausted.
__global__ void __launch_bounds__(kModelThreads)
    t1_model_wide_kernel(const bwc_float *__restrict__ work, const CbDev *__restrict__ cbs,
                    uint32_t ncb, const SbDev *__restrict__ sbs, T1EncOut out,
                    const uint32_t *__restrict__ order, uint32_t *queue, uint32_t stage_cap) {
  if (!queue) {
    if (blockIdx.x < ncb)
      model_codeblock(work, cbs, sbs, out, order ? order[blockIdx.x] : blockIdx.x, stage_cap);
    return;
  }
  __shared__ uint32_t s_next;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t i = s_next;
    __syncthreads();   // every thread has read s_next before it is overwritten
    if (i >= ncb) return;
    model_codeblock(work, cbs, sbs, out, order ? order[i] : i, stage_cap);
    __syncthreads();
  }
}

// ---- the CUDA block behind t1_model.cuh -----------------------------------------------------

struct DevBlock {
  int tid;
  t1::ModelShared *sm;
  __device__ __forceinline__ void sync() { __syncthreads(); }
  __device__ __forceinline__ int sync_or(int v) { return __syncthreads_or(v); }
  __device__ __forceinline__ uint32_t scan(uint32_t v, uint32_t *total) {
    const int lane = tid & 31, w = tid >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sm->wsum[w] = x;
    __syncthreads();
    uint32_t base = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < t1::kModelBlock / 32; ++i) {
      const uint32_t s = sm->wsum[i];
      base += (i < w) ? s : 0u;
      tot += s;
    }
    __syncthreads();
    *total = tot;
    return base + x - v;
  }
  __device__ __forceinline__ uint32_t reduce_max(uint32_t v) {
    v = __reduce_max_sync(0xffffffffu, v);
    if ((tid & 31) == 0) sm->wsum[tid >> 5] = v;
    __syncthreads();
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < t1::kModelBlock / 32; ++i) m = max(m, sm->wsum[i]);
    __syncthreads();
    return m;
  }
  __device__ __forceinline__ void add(long long *p, long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0 && v) atomicAdd(reinterpret_cast<unsigned long long *>(p), (unsigned long long)v);
  }
  __device__ __forceinline__ unsigned long long reserve(unsigned long long *c, unsigned long long n) {
    return atomicAdd(c, n);
  }
  __device__ __forceinline__ void copy16(uint8_t *dst, const uint8_t *src, uint32_t n16) {
    for (uint32_t i = (uint32_t)tid; i < n16; i += t1::kModelBlock)
      reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
  }
  __device__ __forceinline__ void or_flag(uint32_t *f, uint32_t v) { atomicOr(f, v); }
};

constexpr size_t kModelSharedBytes = (sizeof(t1::ModelShared) + 15) & ~size_t(15);

// Context modelling of codeblocks up to 4096 stripe columns.  Without a queue, CTA i models
// codeblock order[i] (or i); with a queue it is persistent over the device work queue.
__global__ void __launch_bounds__(t1::kModelBlock)
    t1_model_kernel(const bwc_float *__restrict__ work, const CbDev *__restrict__ cbs,
                    uint32_t ncb, const SbDev *__restrict__ sbs, T1EncOut out,
                    const uint32_t *__restrict__ order, uint32_t *queue) {
  extern __shared__ __align__(16) uint8_t smem16[];
  t1::ModelShared &sm = *reinterpret_cast<t1::ModelShared *>(smem16);
  uint8_t *stage = smem16 + kModelSharedBytes;
  DevBlock blk{(int)threadIdx.x, &sm};
  __shared__ uint32_t s_next;
  for (;;) {
    uint32_t i = blockIdx.x;
    if (queue) {
      if (threadIdx.x == 0) s_next = atomicAdd(queue, 1u);
      __syncthreads();
      i = s_next;
      __syncthreads();   // every thread has read s_next before it is overwritten
    }
    if (i >= ncb) return;
    const uint32_t c = order ? order[i] : i;
    const CbDev cb = cbs[c];
    const SbDev sb = sbs[cb.sb];
    t1::model_codeblock(blk, sm, stage, work, cb, sb, out, c, &dev::c_sig2ctx[0][0],
                        dev::c_sig2xi, dev::c_xi2cont);
    __syncthreads();   // shared memory is reused by the next codeblock
    if (!queue) return;
  }
}

// ---- MQ coding, truncation lengths, convex hull ----------------------------------------------

// Codes the codeblocks of queue positions [0, nslots): order[slot], or slot without an order.
__global__ void __launch_bounds__(kMqThreads) t1_mq_kernel(const CbDev *__restrict__ cbs,
                                                           uint32_t nslots,
                                                           const SbDev *__restrict__ sbs,
                                                           T1EncOut out, uint32_t lanes,
                                                           const uint32_t *__restrict__ order) {
  __shared__ uint32_t tbl[94];
  // context slots, [context][thread]: every lane of a warp hits its own bank
  __shared__ uint32_t slots[dev::kCtxTotal][kMqThreads];
  for (int i = threadIdx.x; i < 94; i += blockDim.x) tbl[i] = dev::c_mq_states[i];
  __syncthreads();
  // Lanes beyond `lanes`, past the last codeblock, or whose symbol stream did not fit the arena
  // (the host retries those with a larger one) have nothing to code.
  const bool lane_used = threadIdx.x < lanes;
  const uint32_t slot = blockIdx.x * lanes + (lane_used ? threadIdx.x : 0u);
  if (!lane_used || slot >= nslots) return;
  const uint32_t c = order ? order[slot] : slot;
  const int K = out.K[c];
  if (K == 0 || (out.flags[c] & 8u)) return;
  const CbDev cb = cbs[c];
  const SbDev sb = sbs[cb.sb];
  const int Z = out.Z[c];
  const uint64_t pbase = (uint64_t)c * kMaxPasses;
  uint64_t *snaps = out.snaps + pbase * 2;
  t1::MqState e{0x8000u, 0u, 0u, 12, -1};
  t1::ByteSink bo{out.bytes + cb.out_off, cb.out_cap, 0u};
  t1::mq_code_stream(e, bo, out.symbols + out.pass_off[pbase], out.pass_count + pbase, Z, tbl,
                     &slots[0][threadIdx.x], kMqThreads, snaps);
  uint32_t smin, smax;
  t1::t1_finish(e, bo, K, Z, snaps, out.dmse + pbase, sb.gain_step2, out.L + pbase,
                out.S + (uint64_t)c * (kMaxPasses + 1), &smin, &smax);
  if (smax) {
    atomicMin(&out.slopes[2 * cb.slot], smin);
    atomicMax(&out.slopes[2 * cb.slot + 1], smax);
  }
  out.flags[c] |= bo.flags;
}

// ---- MQ coding in two halves: one producer and one consumer warp per CTA ---------------------
// Warp 0 runs the coder's interval half for `lanes` codeblocks, warp 1 its register half for
// the same codeblocks (t1_mq.cuh).  They meet in a shared-memory ring of kMqRing chunks per
// lane: the producer fills slot k % kMqRing with chunk k's (add, shift) pairs and arrives on the
// slot's FULL barrier; the consumer waits on FULL, applies the pairs and arrives on the slot's
// EMPTY barrier, which the producer waits on before refilling the slot.  Both warps take the
// same number of steps (the longest lane's chunk count), so every barrier completes; nothing
// waits on anything outside the CTA.  At the end the consumer adds the producer's A to each
// pass-end snapshot and computes truncation lengths, hull and slopes.
constexpr int kMqRing = 4;   // chunks in flight per lane; barrier ids 1..2*kMqRing and 15

// named barriers of the two warps (64 threads); the calling warp is converged first, as the
// aligned barrier instructions require
__device__ __forceinline__ void named_sync(int id) {
  __syncwarp();
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(64) : "memory");
}
__device__ __forceinline__ void named_arrive(int id) {
  __syncwarp();
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(64) : "memory");
}

__global__ void __launch_bounds__(64) t1_mq_split_kernel(const CbDev *__restrict__ cbs,
                                                         uint32_t nslots,
                                                         const SbDev *__restrict__ sbs,
                                                         T1EncOut out, uint32_t lanes,
                                                         const uint32_t *__restrict__ order) {
  __shared__ uint32_t tbl[94];
  __shared__ t1::MqSlot slots[dev::kCtxTotal][32];
  __shared__ uint32_t ring[kMqRing][16][32];
  __shared__ uint16_t snapA[kMaxPasses][32];
  for (int i = threadIdx.x; i < 94; i += blockDim.x) tbl[i] = dev::c_mq_states[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t slot = blockIdx.x * lanes + (uint32_t)lane;
  const bool have = (uint32_t)lane < lanes && slot < nslots;
  const uint32_t c = have ? (order ? order[slot] : slot) : 0u;
  const int K = have ? out.K[c] : 0;
  // codeblocks with nothing to code, or whose symbol stream did not fit the arena (the host
  // retries those with a larger one), take part in the barriers only
  const bool active = have && K != 0 && !(out.flags[c] & 8u);
  const int Z = active ? out.Z[c] : 0;
  const uint64_t pbase = (uint64_t)c * kMaxPasses;
  const uint32_t *pcount = out.pass_count + pbase;
  const uint32_t nchunks = active ? t1::stream_chunks(pcount, Z) : 0u;
  const uint32_t nsteps = __reduce_max_sync(0xffffffffu, nchunks);
  if (warp == 0) {
    t1::MqProducer P;
    if (active)
      t1::mq_producer_init(P, out.symbols + out.pass_off[pbase], pcount, Z, tbl,
                           &slots[0][lane], 32);
    for (uint32_t k = 0; k < nsteps; ++k) {
      const int r = (int)(k % kMqRing);
      if (k >= (uint32_t)kMqRing) named_sync(1 + kMqRing + r);
      if (active) t1::mq_produce_chunk(P, &ring[r][0][lane], 32, &snapA[0][lane], 32);
      __threadfence_block();
      named_arrive(1 + r);
    }
    for (uint32_t k = nsteps; k < nsteps + kMqRing; ++k)
      if (k >= (uint32_t)kMqRing) named_sync(1 + kMqRing + (int)(k % kMqRing));
    if (active) t1::mq_producer_passes(P, &snapA[0][lane], 32);
    __threadfence_block();
    named_sync(15);
    return;
  }
  const CbDev cb = cbs[c];
  uint64_t *snaps = out.snaps + pbase * 2;
  t1::MqConsumer Q;
  if (active) t1::mq_consumer_init(Q, pcount, Z, out.bytes + cb.out_off, cb.out_cap);
  for (uint32_t k = 0; k < nsteps; ++k) {
    const int r = (int)(k % kMqRing);
    named_sync(1 + r);
    if (active) t1::mq_consume_chunk(Q, &ring[r][0][lane], 32, snaps);
    named_arrive(1 + kMqRing + r);
  }
  if (active) {
    t1::mq_consumer_passes(Q, snaps);
    t1::mq_consumer_overflow(Q);
  }
  named_sync(15);
  if (!active) return;
  for (int p = 0; p < Z; ++p) snaps[2 * p] |= (uint64_t)snapA[p][lane] << 48;
  const SbDev sb = sbs[cb.sb];
  uint32_t smin, smax;
  t1::t1_finish(Q.e, Q.bo, K, Z, snaps, out.dmse + pbase, sb.gain_step2, out.L + pbase,
                out.S + (uint64_t)c * (kMaxPasses + 1), &smin, &smax);
  if (smax) {
    atomicMin(&out.slopes[2 * cb.slot], smin);
    atomicMax(&out.slopes[2 * cb.slot + 1], smax);
  }
  out.flags[c] |= Q.bo.flags;
}

// MQ launch over queue positions [0, n) of `order`: the split kernel (default) or the
// one-warp lane coder (BWC_B200_MQ_SPLIT=0)
void launch_mq(const CbDev *cbs, uint32_t n, const SbDev *sbs, const T1EncOut &out,
               uint32_t lanes, const uint32_t *order, cudaStream_t s) {
  static const bool split = [] {
    const char *v = getenv("BWC_B200_MQ_SPLIT");
    return !(v && v[0] == '0');
  }();
  if (split)
    t1_mq_split_kernel<<<(n + lanes - 1) / lanes, 64, 0, s>>>(cbs, n, sbs, out, lanes, order);
  else
    t1_mq_kernel<<<(n + lanes - 1) / lanes, kMqThreads, 0, s>>>(cbs, n, sbs, out, lanes, order);
}

}  // namespace

// Per-thread symbol staging slice of the wide modelling kernel: 10 symbols for each of the
// thread's columns plus 4 (a pass yields at most 10 per column -- cleanup in run mode: run, two
// position, one sign, three samples of two -- and 4 segmentation symbols), kept while the
// whole block's slices fit in 48 KB; 0 (count the symbols first, then write them) above that.
uint32_t t1_model_stage_cap(uint32_t max_cols) {
  const uint32_t cpt = (max_cols + kModelThreads - 1) / kModelThreads;
  const uint32_t cap = (cpt * 10 + 4 + 3) & ~3u;
  return ((size_t)cap * kModelThreads <= 48 * 1024) ? cap : 0u;
}

static size_t wide_smem(uint32_t max_cols) {
  return (size_t)max_cols * 3 + (size_t)kModelThreads * t1_model_stage_cap(max_cols);
}

// dynamic shared memory of the modelling kernel that runs for codeblocks of up to max_cols
// stripe columns
size_t t1_model_smem(uint32_t max_cols) {
  if (max_cols <= t1::kModelMaxCols) return kModelSharedBytes + t1::kStageBytes;
  return wide_smem(max_cols);
}

// scratch bytes of one codeblock of ncols stripe columns (bit planes of either modelling kernel)
uint64_t t1_scratch_bytes(uint64_t ncols) {
  const uint64_t wide = ncols * (2 + kPrecBit + 1);
  const uint64_t narrow = t1::model_plane_bytes(ncols);
  return ((wide > narrow ? wide : narrow) + 15) & ~15ull;
}

// Codeblocks per MQ warp, the rule used when the autotuner has no entry.  Each lane runs one
// codeblock's coder, a long dependent chain; the per-decision code is straight-line, so the lanes
// of a warp stay converged and a warp codes up to 32 chains for the cost of one.  The rule packs
// codeblocks until there is about one warp per scheduler (148 SMs x 4), where each chain's
// latency, not the issue rate, sets the time.
uint32_t mq_lanes_per_warp(uint32_t ncb) {
  const uint32_t target_warps = (uint32_t)dev::kNumSMs * 4;
  uint32_t lanes = 1;
  while (lanes < 32 && ncb / lanes > target_warps) lanes *= 2;
  return lanes;
}

// ---- autotuner: codeblocks per MQ warp ------------------------------------------------------
// mq_lanes_per_warp is a rule measured on one B200 workload.  The first time a GPU model sees a
// codeblock-count class (the count's bit length) it times the MQ kernel with the candidate lane
// counts around the rule's -- on the real symbol streams; the kernel reads only the streams and
// the model kernel's per-pass records and rewrites all of its outputs, so every run produces the
// same results -- and keeps the fastest for that class.  Results live for the process and, with
// BWC_B200_TUNE_FILE set, in that file (one "gpu-name class lanes" line each), so later
// processes start tuned.  BWC_B200_AUTOTUNE=0 keeps the rule.
namespace {

std::mutex g_tune_mutex;
std::map<std::string, uint32_t> g_tuned;   // "gpu-name/class" -> lanes
bool g_tune_loaded = false;

std::string tune_key(uint32_t ncb) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  std::string name = "gpu";
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) name = prop.name;
  for (char &ch : name)
    if (ch == ' ') ch = '_';
  int cls = 0;
  while ((ncb >> cls) > 1) ++cls;
  return name + "/" + std::to_string(cls);
}

void load_tune_file_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char *path = getenv("BWC_B200_TUNE_FILE");
  if (!path) return;
  FILE *f = fopen(path, "r");
  if (!f) return;
  char key[256];
  unsigned lanes = 0;
  while (fscanf(f, "%255s %u", key, &lanes) == 2)
    if (lanes >= 1 && lanes <= 32) g_tuned[key] = lanes;
  fclose(f);
}

// Side streams of the phased tier-1 launch, one set per device, created on first use and kept.
constexpr int kT1Phases = 4;   // at most 8 (T1LaunchTimes)
std::mutex g_phase_mutex;
cudaStream_t g_phase_streams[64][kT1Phases] = {};

bool phase_streams(cudaStream_t *out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  std::lock_guard<std::mutex> lock(g_phase_mutex);
  for (int i = 0; i < kT1Phases; ++i) {
    if (!g_phase_streams[dev][i] &&
        cudaStreamCreateWithFlags(&g_phase_streams[dev][i], cudaStreamNonBlocking) != cudaSuccess) {
      g_phase_streams[dev][i] = nullptr;
      cudaGetLastError();
      return false;
    }
    out[i] = g_phase_streams[dev][i];
  }
  return true;
}

}  // namespace

// Context modelling, then MQ coding, on `s` (phased across side streams for large counts).
void launch_t1_encode(const bwc_float *work, const CbDev *cbs, uint32_t ncb, const SbDev *sbs,
                      const T1EncOut &out, uint32_t max_cols, cudaStream_t s,
                      const uint32_t *order, uint32_t *queue, cudaEvent_t after_model,
                      T1LaunchTimes *mq_times) {
  if (!ncb) return;
  const size_t smem = t1_model_smem(max_cols);
  const bool narrow = max_cols <= t1::kModelMaxCols;
  // The MQ launches of earlier phases run beside the later phases' modelling for tens of
  // milliseconds.  With the largest shared-memory carveout for all tier-1 kernels, an SM holding
  // MQ CTAs still has room for modelling CTAs, which otherwise waited for those MQ CTAs to end
  // (tier-1 stage at 512^3 between 91 and 241 ms from call to call, by how the CTAs happened to
  // be placed).
  // (function attributes are per device: set on every call, like the dynamic smem size)
  cudaFuncSetAttribute(t1_model_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(t1_model_wide_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(t1_mq_split_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(t1_mq_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutMaxShared);
  if (narrow)
    cudaFuncSetAttribute(t1_model_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  else
    cudaFuncSetAttribute(t1_model_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  unsigned resident = ncb;
  if (queue) {
    // persistent: as many CTAs as fit on the GPU at once
    int dev = 0, sms = dev::kNumSMs, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (narrow)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_model_kernel, t1::kModelBlock, smem);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_model_wide_kernel, kModelThreads, smem);
    resident = (unsigned)std::max(1, sms * std::max(1, per_sm));
  }
  auto model = [&](const uint32_t *ord, uint32_t n, uint32_t *q) {
    const unsigned grid = q ? std::min<unsigned>(n, resident) : n;
    if (q) cudaMemsetAsync(q, 0, sizeof(uint32_t), s);
    if (narrow)
      t1_model_kernel<<<grid, t1::kModelBlock, smem, s>>>(work, cbs, n, sbs, out, ord, q);
    else
      t1_model_wide_kernel<<<grid, kModelThreads, smem, s>>>(work, cbs, n, sbs, out, ord, q,
                                                             t1_model_stage_cap(max_cols));
  };
  const uint32_t rule = mq_lanes_per_warp(ncb);
  uint32_t lanes = rule;
  bool tune = false;
  std::string key;
  const char *at = getenv("BWC_B200_AUTOTUNE");
  if (ncb >= 64 && !(at && at[0] == '0')) {
    key = tune_key(ncb);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    load_tune_file_locked();
    auto it = g_tuned.find(key);
    if (it != g_tuned.end())
      lanes = it->second;
    else
      tune = true;
  }
  // Phased: the work order is largest first, and a codeblock's MQ chain is long, so the
  // codeblocks are modelled in phases (the first 1/64 of the order, then 3/64, 3/16, 3/4), and
  // each phase's MQ kernel runs on a side stream as soon as that phase is modelled, beside the
  // modelling of the later phases.  No kernel waits on another: each side stream waits, by a
  // stream event, for the modelling launch it depends on; the main stream then waits for all.
  cudaStream_t side[kT1Phases];
  const bool phased = order && queue && ncb >= 2048 && phase_streams(side);
  if (!phased) {
    model(order, ncb, queue);
    if (after_model) cudaEventRecord(after_model, s);
    if (mq_times) cudaEventRecord(mq_times->start[0], s);
    launch_mq(cbs, ncb, sbs, out, lanes, order, s);
    if (mq_times) {
      cudaEventRecord(mq_times->end[0], s);
      mq_times->n = 1;
    }
  } else {
    const uint32_t bound[kT1Phases + 1] = {0, ncb / 64, ncb / 16, ncb / 4, ncb};
    cudaEvent_t modelled[kT1Phases], coded[kT1Phases];
    for (int i = 0; i < kT1Phases; ++i) {
      cudaEventCreateWithFlags(&modelled[i], cudaEventDisableTiming);
      cudaEventCreateWithFlags(&coded[i], cudaEventDisableTiming);
    }
    // The phases' modelling launches take one CTA per codeblock (the order's slice, largest
    // first) rather than a persistent grid on the work queue: a persistent kernel ends only when
    // its last CTA has been scheduled, and beside the earlier phases' long MQ launches that CTA
    // sometimes waited for them (512^3: modelling end 28 ms in most calls, up to 112 ms in some;
    // one CTA per codeblock: 28-44 ms, tier-1 93-105 ms against 92-178 ms).
    for (int i = 0; i < kT1Phases; ++i) {
      const uint32_t n = bound[i + 1] - bound[i];
      model(order + bound[i], n, nullptr);
      cudaEventRecord(modelled[i], s);
      cudaStreamWaitEvent(side[i], modelled[i], 0);
      if (mq_times) cudaEventRecord(mq_times->start[i], side[i]);
      launch_mq(cbs, n, sbs, out, lanes, order + bound[i], side[i]);
      if (mq_times) cudaEventRecord(mq_times->end[i], side[i]);
      cudaEventRecord(coded[i], side[i]);
    }
    if (mq_times) mq_times->n = kT1Phases;
    if (after_model) cudaEventRecord(after_model, s);
    for (int i = 0; i < kT1Phases; ++i) {
      cudaStreamWaitEvent(s, coded[i], 0);
      cudaEventDestroy(modelled[i]);   // released once the work that uses it has completed
      cudaEventDestroy(coded[i]);
    }
  }
  if (!tune) return;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  uint32_t best_lanes = rule;
  for (uint32_t cand = std::max(1u, rule / 4); cand <= std::min(32u, rule * 4); cand *= 2) {
    cudaEventRecord(e0, s);
    launch_mq(cbs, ncb, sbs, out, cand, order, s);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      best_lanes = cand;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tuned[key] = best_lanes;
  if (const char *path = getenv("BWC_B200_TUNE_FILE")) {
    if (FILE *f = fopen(path, "a")) {
      fprintf(f, "%s %u\n", key.c_str(), best_lanes);
      fclose(f);
    }
  }
}

extern "C" int bwc_b200_mq_lanes(uint32 ncb) {
  if (!ncb) return 0;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  load_tune_file_locked();
  auto it = g_tuned.find(tune_key(ncb));
  return (int)(it != g_tuned.end() ? it->second : mq_lanes_per_warp(ncb));
}

}  // namespace bwcb
