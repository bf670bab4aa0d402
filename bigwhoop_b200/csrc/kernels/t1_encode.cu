// EBCOT tier-1 encoder: quantisation, bit-plane coding passes, MQ coding, minimal truncation
// lengths and convex-hull rate-distortion slopes.
//
// Reference: cblkcopy_forward (tier1.c:526-729), the three coding passes (tier1.c:962-1511),
// encode_codeblock (tier1.c:2303-2588), the MQ coder (mq.c:85-127, :328-556, :587-759,
// :1151-1175), slope2log and compute_convex_hull (tier1.c:2100-2267).
//
// Two kernels.
//
// t1_model_kernel -- one CTA per codeblock.  Quantises the codeblock into bit planes (global
// scratch), then runs every coding pass over all stripe columns of the codeblock at once and
// writes the pass's (context, decision) symbols, in the reference's scan order, into the
// codeblock's symbol stream.  Contexts only couple samples of the same slice, and within a pass
// a column's outcome depends on its left and upper neighbours' state after the pass and on the
// right and lower neighbours' state before it:
//   * magnitude refinement: all contexts use pre-pass state;
//   * cleanup: a sample's significance after the pass equals (significant | bit) for every
//     sample the pass visits, so every neighbour's post-pass state is known in closed form;
//   * significance propagation: a sample is visited only next to a significant sample, so
//     significance spreads through the pass.  The CTA iterates "column outcome given the
//     current estimates of its left/upper neighbours' outcomes" to a fixed point; the outcome
//     is monotone in the neighbours' significance, so the iteration climbs from the pre-pass
//     state to the sequential result, which is the unique fixed point (dependencies point
//     backwards in scan order).
// Each thread generates its columns' symbols once, into its own shared-memory slice; a
// CTA-wide prefix sum of the counts places them in the pass's arena chunk, and each thread
// copies its slice there (without the slices -- codeblocks over 4608 stripe columns -- the
// symbols are counted first and written in a second run).  Per pass the kernel records the
// symbol count and the distortion decrease.
//
// t1_mq_kernel -- one lane per codeblock.  Runs the MQ arithmetic coder over the codeblock's
// symbol stream (the only part that is inherently sequential), records the coder state at the
// end of every pass, terminates, derives the minimal truncation length of every pass, builds
// the convex hull and the 16-bit log slopes.  A warp holds 1 to 32 codeblocks, each lane with
// its own loop (mq_lanes_per_warp, or the autotuned count).
//
// Stripe-column state (shared memory, one byte each): lo = significance | sign << 4 (read by
// neighbours), hi = visited-in-significance-pass | refined << 4 (owner only).  Bit planes: one
// byte per stripe column per plane, the column's four bits in the low nibble, row 0 at bit 3.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "bwc_b200.h"
#include "device_common.cuh"
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
  __shared__ uint64_t s_base;
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
  __syncthreads();   // planes and column states are read across threads from here on
  if (tid == 0) {
    out.K[c] = (uint8_t)K;
    out.Z[c] = (uint8_t)(3 * K - 2);
  }
  // Every pass's symbols go to their own 16-byte aligned chunk of the shared arena, reserved
  // once the pass's symbol count is known; a full arena marks the codeblock for a retry.
  auto reserve = [&](uint32_t total) -> uint8_t * {
    if (tid == 0) {
      const uint64_t need = ((uint64_t)total + 15) & ~15ull;
      const uint64_t base = atomicAdd(out.sym_used, (unsigned long long)need);
      s_ok = (base + need <= out.sym_cap) ? 1u : 0u;
      s_base = base;
      if (!s_ok) out.flags[c] |= 8u;
    }
    __syncthreads();
    return s_ok ? out.symbols + s_base : nullptr;
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
}

// Kernel 1.  Without a queue, CTA i models codeblock order[i] (or i).  With a queue it is
// persistent: every CTA takes the next position of the device work queue (an atomic counter
// over `order`, largest codeblocks first) until the list is exhausted.
__global__ void __launch_bounds__(kModelThreads)
    t1_model_kernel(const bwc_float *__restrict__ work, const CbDev *__restrict__ cbs,
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

// ---- kernel 2: MQ coding, truncation lengths, convex hull ------------------------------------

// MQ encoder state (mq.c:68-110)
struct Mq {
  uint32_t A, C, T;
  int32_t t;
  int32_t L;
};

struct ByteOut {
  uint8_t *out;
  uint32_t cap;
  uint32_t flags;
};

__device__ __forceinline__ void put_byte(const Mq &e, ByteOut &bo) {
  if (e.L >= 0) {
    if ((uint32_t)e.L < bo.cap) bo.out[e.L] = (uint8_t)e.T; else bo.flags |= 1u;
  }
}

// transfer_byte (mq.c:85-127), due now (t == 0)
__device__ __forceinline__ void mq_transfer(Mq &e, ByteOut &bo) {
  if (e.T != 0xFF && (e.C & 0x8000000u)) {
    e.T++;
    e.C &= 0x7FFFFFFu;
  }
  put_byte(e, bo);
  e.L++;
  if (e.T == 0xFF) {
    e.T = (e.C >> 20) & 0xFF;
    e.C &= 0xFFFFFu;
    e.t += 7;
  } else {
    e.T = (e.C >> 19) & 0xFF;
    e.C &= 0x7FFFFu;
    e.t += 8;
  }
}

__device__ void mq_terminate(Mq &e, ByteOut &bo) {
  // mq_termination (mq.c:706-759)
  int n = 12 - e.t;
  e.C <<= e.t;
  e.t = 0;
  while (n > 0) {
    mq_transfer(e, bo);
    n -= e.t;
    e.C <<= e.t;
    e.t = 0;
  }
  mq_transfer(e, bo);
}

// Minimal number of bytes that decode a pass correctly, from the coder state at its end and the
// bytes emitted later (mq.c:587-675; the single-precision build uses 32-bit split arithmetic).
// Bytes at or beyond `cap` read as zero (the reference's buffer is zero-filled past its data).
__device__ int64_t truncation_length(uint32_t A, uint32_t C, int32_t t, uint32_t T, int64_t L,
                                     const uint8_t *p, uint32_t cap, uint32_t *bad) {
  auto b = [&](int64_t i) -> uint32_t { return (i >= 0 && i < (int64_t)cap) ? p[i] : 0u; };
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
    const int32_t buff = (L >= 0) ? (int32_t)b(L) : 0;
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
    const int64_t buff = (L >= 0) ? (int64_t)b(L) : 0;
    L++;
    Cr -= buff << (35 - s);
    CAr -= buff << (35 - s);
    Cr = (int64_t)((uint64_t)Cr << s);
    CAr = (int64_t)((uint64_t)CAr << s);
    s = (buff == 0xFF) ? 7 : 8;
  }
#endif
  if (L > 0 && b(L - 1) == 0xFF) L--;
  while (L > 1 && b(L - 2) == 0xFF && b(L - 1) == 0x7F) L -= 2;
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

__global__ void __launch_bounds__(kMqThreads) t1_mq_kernel(const CbDev *__restrict__ cbs,
                                                           uint32_t ncb,
                                                           const SbDev *__restrict__ sbs,
                                                           T1EncOut out, uint32_t lanes,
                                                           const uint32_t *__restrict__ order) {
  __shared__ uint32_t tbl[94];
  // context states, [context][thread]: every lane of a warp hits its own bank
  __shared__ uint32_t ctx_all[dev::kCtxTotal][kMqThreads];
  for (int i = threadIdx.x; i < 94; i += blockDim.x) tbl[i] = dev::c_mq_states[i];
  __syncthreads();
  // Lanes beyond `lanes`, past the last codeblock, or whose symbol stream did not fit the arena
  // (the host retries those with a larger one) have nothing to code.
  const bool lane_used = threadIdx.x < lanes;
  const uint32_t slot = blockIdx.x * lanes + (lane_used ? threadIdx.x : 0u);
  const uint32_t c = (slot < ncb) ? (order ? order[slot] : slot) : ncb;
  const uint32_t cc = (c < ncb) ? c : 0u;
  const int K = (lane_used && c < ncb) ? out.K[c] : 0;
  const bool live = (K != 0) && !(out.flags[cc] & 8u);
  const CbDev cb = cbs[cc];
  const SbDev sb = sbs[cb.sb];
  const int Z = live ? out.Z[c] : 0;
  // context slots hold their current state's table entry
  uint32_t *ctx = &ctx_all[0][threadIdx.x];   // context k at ctx[k * kMqThreads]
  for (int i = 0; i < dev::kCtxTotal; ++i)
    ctx[i * kMqThreads] = tbl[dev::mq_initial_state(i)];
  const uint32_t *pcount = out.pass_count + (uint64_t)cc * kMaxPasses;
  const uint64_t *poff = out.pass_off + (uint64_t)cc * kMaxPasses;
  uint64_t *snaps = out.snaps + (uint64_t)cc * kMaxPasses * 2;
  int64_t *dmse = out.dmse + (uint64_t)cc * kMaxPasses;
  ByteOut bo{out.bytes + cb.out_off, cb.out_cap, 0u};
  Mq e{0x8000u, 0u, 0u, 12, -1};
  auto snapshot = [&](int p) {
    snaps[2 * p] = ((uint64_t)e.A << 48) | ((uint64_t)(e.T & 0xFF) << 40) |
                   ((uint64_t)(uint8_t)e.t << 32) | (uint64_t)(uint32_t)e.C;
    snaps[2 * p + 1] = (uint64_t)(int64_t)e.L;
  };
  if (!live) return;
  // Each lane codes its codeblock on its own: passes in order, the state snapshot at the end of
  // each.  A pass's symbols are read a 32-bit word (four symbols) at a time, two words ahead.
  // Per symbol (mq_bit_encode, mq.c:478-556): the common case -- the more probable symbol with
  // the interval staying >= 0x8000 -- is a subtraction and an addition; otherwise the context
  // moves to its next state, the interval renormalises (a plain shift unless a byte falls due
  // on the way, mq.c:85-127 then) and the coder state advances.  The next symbol's context
  // entry is read while the current symbol is coded; a context the current symbol just changed
  // overrides it.
  auto code = [&](uint32_t sym, uint32_t ent, uint32_t nk, uint32_t &nent) {
    const uint32_t pq = ent & 0xFFFF;
    const uint32_t A1 = e.A - pq;
    const bool is_mps = ((sym ^ (ent >> 16)) & 1) == 0;
    if (is_mps && A1 >= 0x8000u) {
      e.A = A1;
      e.C += pq;
      return;
    }
    const bool small = A1 < pq;
    e.C += (is_mps != small) ? pq : 0u;
    e.A = (is_mps == small) ? pq : A1;
    const uint32_t k = sym >> 1;
    const uint32_t ne = tbl[is_mps ? (ent >> 17) & 0x7F : (ent >> 24) & 0x7F];
    ctx[k * kMqThreads] = ne;
    if (nk == k) nent = ne;
    int sh = __clz(e.A) - 16;   // shifts until A >= 0x8000 (at least one)
    if (sh < e.t) {
      e.A <<= sh;
      e.C <<= sh;
      e.t -= sh;
      return;
    }
    do {   // shift up to each due transfer, transfer, continue
      const int s1 = min(sh, e.t);
      e.A <<= s1;
      e.C <<= s1;
      e.t -= s1;
      sh -= s1;
      if (e.t == 0) mq_transfer(e, bo);
    } while (sh > 0);
  };
  for (int p = 0; p < Z; ++p) {
    const uint32_t n = pcount[p];
    if (n) {
      // the pass's chunk holds at least (n + 3) / 4 words
      const uint32_t *src = reinterpret_cast<const uint32_t *>(out.symbols + poff[p]);
      const uint32_t nw = (n + 3) >> 2;
      uint32_t w = src[0];
      uint32_t wn = (nw > 1) ? src[1] : 0u;
      uint32_t ent = ctx[((w & 0xFF) >> 1) * kMqThreads];
      uint32_t left = n;
      for (uint32_t q = 0; q < nw; ++q) {
        const uint32_t wc = w;
        w = wn;
        wn = (q + 2 < nw) ? src[q + 2] : 0u;
        const uint32_t cnt = min(left, 4u);
        left -= cnt;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          if ((uint32_t)jj < cnt) {
            const uint32_t sym = (wc >> (8 * jj)) & 0xFF;
            const uint32_t nsym = (jj < 3) ? (wc >> (8 * (jj + 1))) & 0xFF : (w & 0xFF);
            // past the pass's last symbol the next byte is padding: clamp its context index
            const uint32_t nk = min(nsym >> 1, (uint32_t)dev::kCtxTotal - 1);
            uint32_t nent = ctx[nk * kMqThreads];
            code(sym, ent, nk, nent);
            ent = nent;
          }
        }
      }
    }
    snapshot(p);
  }
  mq_terminate(e, bo);
  for (int i = 0; i < 16; ++i) {
    const int64_t q = (int64_t)e.L + i;
    if (q >= 0 && (uint64_t)q < bo.cap) bo.out[q] = 0;
  }
  // truncation lengths
  uint32_t *Lout = out.L + (uint64_t)c * kMaxPasses;
  uint32_t bad = 0;
  for (int j = 0; j < Z; ++j) {
    const uint64_t s0 = snaps[2 * j];
    const int64_t Ls = (int64_t)snaps[2 * j + 1];
    Lout[j] = (uint32_t)truncation_length((uint32_t)(s0 >> 48), (uint32_t)s0,
                                          (int32_t)(int8_t)((s0 >> 32) & 0xFF),
                                          (uint32_t)((s0 >> 40) & 0xFF), Ls, bo.out, bo.cap, &bad);
  }
  if (bad) bo.flags |= 4u;
  // convex hull (scratch: slopes and hull stack overwrite the snapshots; dmse stays as it is,
  // so the kernel can run again on the same symbol streams)
  double *lambda = reinterpret_cast<double *>(snaps);
  uint8_t *hull = reinterpret_cast<uint8_t *>(snaps + kMaxPasses + 1);
  double scale0 = sb.gain_step2;
  scale0 = dev::fmul(scale0, ldexp(1.0, 2 * K));
  scale0 = dev::fdiv(scale0, 65536.0);
  // distortion decrease of pass q in the reference's weighting: the weight is scale0 for the
  // first plane and a quarter less per plane below (exact: powers of two, no subnormals);
  // pass 0 codes plane K-1, passes 1-3 plane K-2, and so on
  auto mse_of = [&](int q) -> double {
    return dev::fmul(__ll2double_rn(dmse[q]), ldexp(scale0, -2 * ((q + 2) / 3)));
  };
  for (int i = 0; i <= Z; ++i) lambda[i] = 0.0;
  for (int i = 0; i < Z; ++i) hull[i] = 0;
  lambda[0] = 18446744073709551616.0;
  int h = 0, hlast = 0;
  for (int i = 0; i < Z; ++i) {
    double dD = 0.0;
    for (int q = hlast; q <= i; ++q) dD = dev::fadd(dD, mse_of(q));
    uint64_t dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
    if (dD > 0) {
      while (dD >= dev::fmul(lambda[hlast], __ull2double_rn(dL))) {
        lambda[hlast] = 0;
        if (h == 0) {
          // the reference would read below its hull stack here
          bo.flags |= 2u;
          break;
        }
        h--;
        hlast = hull[h];
        dD = 0.0;
        for (int q = hlast; q <= i; ++q) dD = dev::fadd(dD, mse_of(q));
        dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
      }
      h++;
      hlast = i + 1;
      hull[h] = (uint8_t)hlast;
      if (dL == 0)
        lambda[hlast] = (dD < 0) ? -1.0 : (dD == 0 ? 0.0 : 18446744073709551616.0);
      else
        lambda[hlast] = dev::fdiv(dD, __ull2double_rn(dL));
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
    atomicMin(&out.slopes[2 * cb.slot], smin);
    atomicMax(&out.slopes[2 * cb.slot + 1], smax);
  }
  out.flags[c] |= bo.flags;
}

}  // namespace

// Per-thread symbol staging slice of the modelling kernel: 10 symbols for each of the thread's
// columns plus 4 (a pass yields at most 10 per column -- cleanup in run mode: run, two
// position, one sign, three samples of two -- and 4 segmentation symbols), kept while the
// whole block's slices fit in 48 KB; 0 (count the symbols first, then write them) above that.
uint32_t t1_model_stage_cap(uint32_t max_cols) {
  const uint32_t cpt = (max_cols + kModelThreads - 1) / kModelThreads;
  const uint32_t cap = (cpt * 10 + 4 + 3) & ~3u;
  return ((size_t)cap * kModelThreads <= 48 * 1024) ? cap : 0u;
}

size_t t1_model_smem(uint32_t max_cols) {
  return (size_t)max_cols * 3 + (size_t)kModelThreads * t1_model_stage_cap(max_cols);
}

// Codeblocks per MQ warp, the rule used when the autotuner has no entry.  Each lane runs one
// codeblock's coder, a long dependent chain, so a warp is latency-bound and its lanes diverge
// (symbol kinds, byte transfers, pass ends); fewer lanes per warp waste less, until the warps'
// instructions saturate the schedulers.  Measured on B200 (FP64, 32x32x16 codeblocks): 1030
// codeblocks code fastest at 1 per warp, 8192 at 4 per warp, i.e. at about three warps per
// scheduler (148 SMs x 4).
uint32_t mq_lanes_per_warp(uint32_t ncb) {
  const uint32_t target_warps = (uint32_t)dev::kNumSMs * 4 * 3;
  uint32_t lanes = 1;
  while (lanes < 32 && ncb / (lanes * 2) >= target_warps) lanes *= 2;
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

}  // namespace

// Context modelling, then MQ coding, on `s`.  (Running the modelling of later codeblocks
// concurrently with the MQ coding of earlier ones was measured slower: the issue-bound modelling
// warps lengthen the latency-bound MQ chains, and the longest chain sets the time.)
void launch_t1_encode(const bwc_float *work, const CbDev *cbs, uint32_t ncb, const SbDev *sbs,
                      const T1EncOut &out, uint32_t max_cols, cudaStream_t s,
                      const uint32_t *order, uint32_t *queue, cudaEvent_t after_model) {
  if (!ncb) return;
  const size_t smem = t1_model_smem(max_cols);
  cudaFuncSetAttribute(t1_model_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  unsigned grid = ncb;
  if (queue) {
    // persistent: as many CTAs as fit on the GPU at once
    int dev = 0, sms = dev::kNumSMs, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_model_kernel, kModelThreads, smem);
    grid = std::min<unsigned>(ncb, (unsigned)std::max(1, sms * std::max(1, per_sm)));
    cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
  }
  t1_model_kernel<<<grid, kModelThreads, smem, s>>>(work, cbs, ncb, sbs, out, order, queue,
                                                    t1_model_stage_cap(max_cols));
  if (after_model) cudaEventRecord(after_model, s);
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
  t1_mq_kernel<<<(ncb + lanes - 1) / lanes, kMqThreads, 0, s>>>(cbs, ncb, sbs, out, lanes, order);
  if (!tune) return;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  uint32_t best_lanes = rule;
  for (uint32_t cand = std::max(1u, rule / 4); cand <= std::min(32u, rule * 4); cand *= 2) {
    cudaEventRecord(e0, s);
    t1_mq_kernel<<<(ncb + cand - 1) / cand, kMqThreads, 0, s>>>(cbs, ncb, sbs, out, cand, order);
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
