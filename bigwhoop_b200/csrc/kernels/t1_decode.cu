// EBCOT tier-1 decoder and dequantiser -- one codeblock per warp.
//
// Reference: decoding passes (tier1.c:1543-2069), decode_codeblock (tier1.c:2624-2787), MQ
// decoder (mq.c:147-173, :846-1029), dequantisation cblkcopy_inverse (tier1.c:767-931).
//
// Decoding is inherently sequential inside a codeblock (every context depends on the bits just
// decoded), so one lane walks the passes while the other lanes wait; the whole warp then
// reconstructs the samples in parallel: value = (magnitude + 0.475 * 2^p) * step with p the
// first undecoded bit plane (one plane lower for samples whose last pass was not reached), sign
// from the decoded sign bit.
//
// t1_decode_kernel (codeblocks up to 4096 stripe columns): the decoder of t1_dec.cuh -- state as
// 64-bit sample masks per 16 columns in shared memory, contexts from per-class tables, decoded
// bits as one mask per plane and 16 columns in global memory, magnitudes rebuilt by bit
// transposes.  t1_decode_wide_kernel (larger codeblocks): column states in shared memory and
// magnitudes accumulated in global memory, one stripe column at a time.
#include <algorithm>

#include "device_common.cuh"
#include "t1_dec.cuh"
#include "t1_tables.cuh"

namespace bwcb {
namespace {

using dev::kCtxMag;
using dev::kCtxRun;
using dev::kCtxSig;
using dev::kCtxUni;

constexpr int kWarpsPerBlock = 4;

struct MqDec {
  uint32_t A, C;
  int32_t t;
  uint32_t T;
  int64_t L, Lmax;
  const uint8_t *b;
};

__device__ __forceinline__ void fill_lsb(MqDec &d) {
  if (d.L == d.Lmax || (d.T == 0xFF && d.b[d.L] > 0x8f)) {
    d.t = 8;
    d.C += 0xFF;
  } else if (d.T == 0xFF) {
    d.t = 7;
    d.T = d.b[d.L];
    d.C += d.T << 1;
    d.L++;
  } else {
    d.t = 8;
    d.T = d.b[d.L];
    d.C += d.T;
    d.L++;
  }
}

// Renormalisation (mq.c decoder): shift A and C left until A >= 0x8000, reading the next byte
// whenever the bit counter t is empty before a shift.  Done in runs of min(shifts left, t)
// shifts, the counter only empties at a run's end, so the bytes come in at the same points as
// one shift at a time.
__device__ __forceinline__ void renorm(MqDec &d) {
  int sh = __clz(d.A) - 16;   // A in [1, 0x7FFF]: at least one shift
  do {
    if (d.t == 0) fill_lsb(d);
    const int s1 = min(sh, d.t);
    d.A = (d.A << s1) & 0xFFFF;
    d.C <<= s1;
    d.t -= s1;
    sh -= s1;
  } while (sh > 0);
}

__device__ __forceinline__ uint32_t mq_decode(MqDec &d, uint8_t *ctx, int k) {
  const uint32_t ent = dev::c_mq_states[ctx[k]];
  const uint32_t p = ent & 0xFFFF;
  uint32_t x = (ent >> 16) & 1;
  d.A = (d.A - p) & 0xFFFF;
  if ((d.C >> 8) >= p) {
    d.C -= p << 8;
    d.C &= 0xFFFFFF;
    if (!(d.A & 0x8000)) {
      if (d.A < p) {
        x = 1 - x;
        ctx[k] = (uint8_t)((ent >> 24) & 0x7F);
      } else {
        ctx[k] = (uint8_t)((ent >> 17) & 0x7F);
      }
      renorm(d);
    }
  } else {
    if (d.A < p) {
      ctx[k] = (uint8_t)((ent >> 17) & 0x7F);
    } else {
      x = 1 - x;
      ctx[k] = (uint8_t)((ent >> 24) & 0x7F);
    }
    d.A = p;
    renorm(d);
  }
  return x;
}

__device__ __forceinline__ uint32_t bit(uint32_t v, int i) { return (i >= 0 && i < 4) ? (v >> i) & 1u : 0u; }

struct Geo {
  uint32_t W, nstripes, nfull, rem, ncols;
};

struct Col {
  uint32_t L, R, U, UL, UR, D, DL, DR;   // sigma | xi << 4 of the neighbours
};

// stripe-column cursor: col = x + W * (j + nstripes * slice), advanced column by column
__device__ __forceinline__ void advance(uint32_t &x, uint32_t &j, const Geo &g) {
  if (++x == g.W) {
    x = 0;
    if (++j == g.nstripes) j = 0;
  }
}

__device__ __forceinline__ Col neighbours(const uint16_t *state, const Geo &g, uint32_t col,
                                          uint32_t x, uint32_t j) {
  Col n{0, 0, 0, 0, 0, 0, 0, 0};
  if (x > 0) n.L = state[col - 1] & 0xFF;
  if (x + 1 < g.W) n.R = state[col + 1] & 0xFF;
  if (j > 0) {
    n.U = state[col - g.W] & 0xFF;
    if (x > 0) n.UL = state[col - g.W - 1] & 0xFF;
    if (x + 1 < g.W) n.UR = state[col - g.W + 1] & 0xFF;
  }
  if (j + 1 < g.nstripes) {
    n.D = state[col + g.W] & 0xFF;
    if (x > 0) n.DL = state[col + g.W - 1] & 0xFF;
    if (x + 1 < g.W) n.DR = state[col + g.W + 1] & 0xFF;
  }
  return n;
}

__device__ __forceinline__ uint32_t sig_index(uint32_t sig, const Col &n, int l, bool full) {
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

__device__ __forceinline__ uint32_t decode_sign(MqDec &d, uint8_t *ctx, uint32_t sig, uint32_t xi,
                                                const Col &n, int l, bool full) {
  const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF, Lx = n.L >> 4, Rx = n.R >> 4;
  const uint32_t xh = bit(Ls, l) | (bit(Rs, l) << 1) | (bit(Lx, l) << 2) | (bit(Rx, l) << 3);
  uint32_t xv = bit(sig, l + 1) | (bit(sig, l - 1) << 1) | (bit(xi, l + 1) << 2) | (bit(xi, l - 1) << 3);
  if (l == 3) {
    xv |= (n.U & 1) | (((n.U >> 4) & 1) << 2);
  } else if (l == 0 && full) {
    xv |= (((n.D >> 3) & 1) << 1) | (((n.D >> 7) & 1) << 3);
  }
  const uint32_t e = dev::c_xi2cont[(dev::c_sig2xi[xh] << 2) | dev::c_sig2xi[xv]];
  return (e >> 7) ^ mq_decode(d, ctx, e & 0x7F);
}

__device__ void dec_sp(MqDec &d, uint8_t *ctx, uint16_t *state, bwc_raw *mag, const Geo &g,
                       uint32_t cls, int b) {
  for (uint32_t col = 0, x = 0, j = 0; col < g.ncols; ++col, advance(x, j, g)) {
    const bool full = j < g.nfull;
    const int lmin = full ? 0 : 4 - (int)g.rem;
    const uint32_t vmask = (0xFu >> lmin) << lmin;
    uint32_t st = state[col];
    uint32_t sig = st & 0xF, xi = (st >> 4) & 0xF, pi = (st >> 8) & 0xF;
    if (((sig ^ 0xF) & vmask) == 0) {
      state[col] = (uint16_t)(st & 0xF0FFu);
      continue;
    }
    const Col n = neighbours(state, g, col, x, j);
    for (int l = 3; l >= lmin; --l) {
      const uint32_t m = 1u << l;
      if (!(sig & m)) {
        const uint32_t ks = sig_index(sig, n, l, full);
        if (ks) {
          if (mq_decode(d, ctx, kCtxSig + dev::c_sig2ctx[cls][ks])) {
            mag[col * 4 + (3 - l)] |= (bwc_raw)1 << b;
            xi |= decode_sign(d, ctx, sig, xi, n, l, full) << l;
            sig |= m;
          }
          pi |= m;
        }
      } else {
        pi &= ~m;
      }
    }
    state[col] = (uint16_t)((st & 0xF000u) | (pi << 8) | (xi << 4) | sig);
  }
}

__device__ void dec_mr(MqDec &d, uint8_t *ctx, uint16_t *state, bwc_raw *mag, const Geo &g, int b) {
  for (uint32_t col = 0, x = 0, j = 0; col < g.ncols; ++col, advance(x, j, g)) {
    const bool full = j < g.nfull;
    const int lmin = full ? 0 : 4 - (int)g.rem;
    const uint32_t vmask = (0xFu >> lmin) << lmin;
    const uint32_t st = state[col];
    const uint32_t sig = st & 0xF, pi = (st >> 8) & 0xF;
    uint32_t delta = (st >> 12) & 0xF;
    const uint32_t todo = sig & ~pi & vmask;
    if (!todo) continue;
    // neighbours only decide the context of a sample's first refinement
    Col n{0, 0, 0, 0, 0, 0, 0, 0};
    if (todo & ~delta) n = neighbours(state, g, col, x, j);
    const uint32_t Ls = n.L & 0xF, Rs = n.R & 0xF;
    for (int l = 3; l >= lmin; --l) {
      const uint32_t m = 1u << l;
      if (todo & m) {
        uint32_t k = kCtxMag;
        if (delta & m) {
          k += 2;
        } else {
          uint32_t any = bit(sig, l + 1) | bit(sig, l - 1) | bit(Ls, l) | bit(Rs, l) |
                         bit(Ls, l + 1) | bit(Ls, l - 1) | bit(Rs, l + 1) | bit(Rs, l - 1);
          if (l == 3) any |= (n.U | n.UL | n.UR) & 1;
          if (l == 0 && full) any |= ((n.D | n.DL | n.DR) >> 3) & 1;
          k += any ? 1 : 0;
        }
        if (mq_decode(d, ctx, k)) mag[col * 4 + (3 - l)] |= (bwc_raw)1 << b;
        delta |= m;
      }
    }
    state[col] = (uint16_t)((st & 0x0FFFu) | (delta << 12));
  }
}

__device__ void dec_cu(MqDec &d, uint8_t *ctx, uint16_t *state, bwc_raw *mag, const Geo &g,
                       uint32_t cls, int b) {
  for (uint32_t col = 0, x = 0, j = 0; col < g.ncols; ++col, advance(x, j, g)) {
    const bool full = j < g.nfull;
    const int lmin = full ? 0 : 4 - (int)g.rem;
    const uint32_t st = state[col];
    uint32_t sig = st & 0xF, xi = (st >> 4) & 0xF;
    const uint32_t pi = (st >> 8) & 0xF;
    const Col n = neighbours(state, g, col, x, j);
    uint32_t bits = 0;
    int r = -1;
    if (full) {
      const uint32_t around = ((n.D | n.DL | n.DR) & 0x8) | ((n.U | n.UL | n.UR) & 0x1) |
                              (n.L & 0xF) | (n.R & 0xF) | sig;
      if (!around) {
        if (mq_decode(d, ctx, kCtxRun)) {
          r = (int)mq_decode(d, ctx, kCtxUni);
          r = (r << 1) + (int)mq_decode(d, ctx, kCtxUni);
          bits |= 0x08u >> r;
        } else {
          r = 4;
        }
      }
    }
    for (int l = 3; l >= lmin; --l) {
      const uint32_t m = 1u << l;
      if (!(sig & m) && !(pi & m)) {
        if (r >= 0) {
          r--;
        } else {
          bits |= mq_decode(d, ctx, kCtxSig + dev::c_sig2ctx[cls][sig_index(sig, n, l, full)]) << l;
        }
        if (bits & m) {
          xi |= decode_sign(d, ctx, sig, xi, n, l, full) << l;
          sig |= m;
        }
      }
    }
    for (int l = 3; l >= 0; --l)
      if (bits & (1u << l)) mag[col * 4 + (3 - l)] |= (bwc_raw)1 << b;
    state[col] = (uint16_t)((st & 0xFF00u) | (xi << 4) | sig);
  }
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    t1_decode_wide_kernel(bwc_float *__restrict__ work, const CbDev *__restrict__ cbs,
                     uint32_t ncb, const SbDev *__restrict__ sbs, const uint8_t *__restrict__ data,
                     const uint8_t *__restrict__ Kin, const uint8_t *__restrict__ Zin,
                     const uint32_t *__restrict__ Lmax, uint32_t erres, bwc_raw *mags,
                     uint32_t *flags, uint32_t state_cap, uint16_t *gstate,
                     uint32_t *work_counter, const uint32_t *__restrict__ order) {
  extern __shared__ unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint8_t *ctx = smem_raw + wib * 32;
  __shared__ int s_bitplane[kWarpsPerBlock], s_pass[kWarpsPerBlock];
  uint16_t *sstate = reinterpret_cast<uint16_t *>(smem_raw + 32 * kWarpsPerBlock) +
                     (size_t)wib * state_cap;
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(work_counter, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= ncb) break;
    if (order) c = order[c];   // the queue position's codeblock (largest coded length first)
    const CbDev cb = cbs[c];
    const SbDev sb = sbs[cb.sb];
    Geo g;
    g.W = cb.w;
    g.nstripes = (cb.h + 3) >> 2;
    g.nfull = cb.h >> 2;
    g.rem = cb.h & 3;
    g.ncols = g.W * g.nstripes * cb.d * cb.nt;
    uint16_t *state = (g.ncols <= state_cap) ? sstate : gstate + (uint64_t)cb.scratch_off;
    if (g.ncols > state_cap && !gstate) {
      if (lane == 0) flags[c] |= 4u;
      continue;
    }
    bwc_raw *mag = mags + cb.scratch_off;
    for (uint32_t i = lane; i < g.ncols; i += 32) state[i] = 0;
    for (uint32_t i = lane; i < g.ncols * 4; i += 32) mag[i] = 0;
    if (lane < dev::kCtxTotal) ctx[lane] = dev::mq_initial_state(lane);
    __syncwarp();
    const int K = Kin[c], Z = Zin[c];
    if (lane == 0) {
      int bitplane = 0, cpass = 0;
      if (Z > 0) {
        MqDec d;
        d.b = data + cb.out_off;
        d.Lmax = Lmax[c];
        d.L = 0;
        d.T = 0;
        d.C = 0;
        d.t = 0;
        d.A = 0;
        fill_lsb(d);
        d.C <<= 8;
        fill_lsb(d);
        d.C <<= 7;
        d.t -= 7;
        d.A = 0x8000;
        int i = 2, j = Z, k = K;
        bool broke = false;
        while (k-- > 0) {
          for (; i < 3; ++i, --j) {
            if (j == 0) {
              broke = true;
              break;
            }
            if (i == 0) dec_sp(d, ctx, state, mag, g, sb.cls, k);
            else if (i == 1) dec_mr(d, ctx, state, mag, g, k);
            else dec_cu(d, ctx, state, mag, g, sb.cls, k);
          }
          if (broke) break;
          if (erres) {
            uint32_t v = mq_decode(d, ctx, kCtxUni) << 3;
            v |= mq_decode(d, ctx, kCtxUni) << 2;
            v |= mq_decode(d, ctx, kCtxUni) << 1;
            v |= mq_decode(d, ctx, kCtxUni);
            if (v != 0x0A) {
              broke = true;
              break;
            }
          }
          i = 0;
        }
        if (!broke) i = 0;
        bitplane = (k > 0) ? k : 0;
        cpass = i;
      }
      s_bitplane[wib] = bitplane;
      s_pass[wib] = cpass;
    }
    __syncwarp();
    const int bitplane = s_bitplane[wib], cpass = s_pass[wib];
    // ---- dequantise into the working buffer ---------------------------------------------------
    const uint64_t sy = cb.sy, sz = cb.sz, st_ = cb.st;
    for (uint32_t q = lane; q < g.ncols * 4; q += 32) {
      const uint32_t col = q >> 2, row = q & 3;
      const bwc_raw m = mag[q];
      if (!m) continue;
      const uint32_t x = col % g.W, sr = col / g.W;
      const uint32_t jj = sr % g.nstripes, sl = sr / g.nstripes;
      const uint32_t y = 4 * jj + row;
      const uint32_t z = sl % cb.d, t = sl / cb.d;
      const uint32_t stw = state[col];
      const uint32_t l = 3 - row;
      const uint32_t pib = (stw >> (8 + l)) & 1, xib = (stw >> (4 + l)) & 1;
      const int shift = bitplane + ((!cpass || pib) ? 0 : 1);
      const float off = __fmul_rn((float)((uint64_t)1 << shift), 0.475f);
      bwc_float f = dev::from_u64_rn((uint64_t)m);
      f = dev::fadd(f, (bwc_float)off);
      f = dev::fmul(f, sb.qt_eff);
      bwc_raw r = dev::as_raw(f) | (xib ? kSignMask : (bwc_raw)0);
      work[cb.base + (cb.x0 + x) + (uint64_t)(cb.y0 + y) * sy + (uint64_t)(cb.z0 + z) * sz +
           (uint64_t)(cb.t0 + t) * st_] = dev::as_float(r);
    }
    __syncwarp();
  }
}

// ---- codeblocks up to 4096 stripe columns ---------------------------------------------------

constexpr int kDecWarps = 4;

struct DecWarpShared {
  t1::u64 sig[256], sgn[256], pi[256], del[256], bits[256];
  uint32_t slot[dev::kCtxTotal + 1];
};

__global__ void __launch_bounds__(kDecWarps * 32)
    t1_decode_kernel(bwc_float *__restrict__ work, const CbDev *__restrict__ cbs, uint32_t ncb,
                     const SbDev *__restrict__ sbs, const uint8_t *__restrict__ data,
                     const uint8_t *__restrict__ Kin, const uint8_t *__restrict__ Zin,
                     const uint32_t *__restrict__ Lmax, uint32_t erres, bwc_raw *mags,
                     uint32_t *flags, uint32_t *work_counter, const uint32_t *__restrict__ order) {
  __shared__ t1::DecTables tabs;
  __shared__ uint32_t tbl[94];
  __shared__ DecWarpShared wsh[kDecWarps];
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    t1::dec_table_entry(tabs, i, &dev::c_sig2ctx[0][0], dev::c_sig2xi, dev::c_xi2cont);
  for (int i = threadIdx.x; i < 94; i += blockDim.x) tbl[i] = dev::c_mq_states[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  DecWarpShared &ws = wsh[wib];
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(work_counter, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= ncb) break;
    if (order) c = order[c];   // the queue position's codeblock (largest coded length first)
    const CbDev cb = cbs[c];
    const SbDev sb = sbs[cb.sb];
    const uint32_t ncols = cb.w * ((cb.h + 3) >> 2) * cb.d * cb.nt;
    if (ncols > t1::kModelMaxCols) {
      if (lane == 0) flags[c] |= 4u;
      continue;
    }
    const int ngroups = (int)((ncols + 15) >> 4);
    const int K = Kin[c], Z = Zin[c];
    t1::u64 *planes = reinterpret_cast<t1::u64 *>(mags + cb.scratch_off);
    int r0 = 0, r1 = 0, r2 = K;
    if (lane == 0) {
      const t1::DecOut res =
          t1::decode_seq(data + cb.out_off, Lmax[c], K, Z, erres != 0, cb.w, cb.h, ncols,
                         (int)sb.cls, ws.sig, ws.sgn, ws.pi, ws.del, ws.bits, ws.slot, tbl, tabs,
                         planes);
      r0 = res.bitplane;
      r1 = res.cpass;
      r2 = res.pmin;
    }
    t1::DecOut res;
    res.bitplane = __shfl_sync(0xffffffffu, r0, 0);
    res.cpass = __shfl_sync(0xffffffffu, r1, 0);
    res.pmin = __shfl_sync(0xffffffffu, r2, 0);
    __syncwarp();
    for (int g = lane; g < ngroups; g += 32)
      t1::dequant_group(g, ngroups, K, res, planes, ws.sgn[g], ws.pi[g], cb, sb.qt_eff, work, cb.w,
                        cb.h, ncols);
    __syncwarp();
  }
}

}  // namespace

// decode scratch (elements of bwc_raw) of one codeblock of ncols stripe columns: its decoded
// bit planes (one 64-bit mask per 16 columns and plane), or the wide kernel's magnitudes
uint64_t t1_decode_scratch_elems(uint64_t ncols) { return ((ncols + 15) / 16) * 64; }

void launch_t1_decode_ex(bwc_float *work, const CbDev *cbs, uint32_t ncb,
                         const SbDev *sbs, const uint8_t *data, const uint8_t *K,
                         const uint8_t *Z, const uint32_t *Lmax, uchar erres, bwc_raw *mags,
                         uint32_t *flags, uint32_t state_cap, uint16_t *gstate,
                         uint32_t *work_counter, int grid, cudaStream_t s,
                         const uint32_t *order, uint32_t max_cols) {
  if (max_cols <= t1::kModelMaxCols) {
    int dev = 0, sms = dev::kNumSMs, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_decode_kernel, kDecWarps * 32, 0);
    const unsigned g = (unsigned)std::max(1, sms * std::max(1, per_sm));
    t1_decode_kernel<<<g, kDecWarps * 32, 0, s>>>(work, cbs, ncb, sbs, data, K, Z, Lmax, erres,
                                                 mags, flags, work_counter, order);
    return;
  }
  const size_t smem = 32 * kWarpsPerBlock + (size_t)state_cap * sizeof(uint16_t) * kWarpsPerBlock;
  cudaFuncSetAttribute(t1_decode_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  t1_decode_wide_kernel<<<grid, kWarpsPerBlock * 32, smem, s>>>(work, cbs, ncb, sbs, data, K, Z,
                                                                Lmax, erres, mags, flags, state_cap,
                                                                gstate, work_counter, order);
}

}  // namespace bwcb
