// Pieces of the tier-1 encoder shared by the CUDA kernels and by the host build of the kernel
// bodies (bigwhoop_b200/csrc/emu, the CPU unit tests of the kernel logic): exactly rounded
// arithmetic in both worlds, the MQ coder's byte output and termination, minimal truncation
// lengths, log slopes and the convex hull of one codeblock.
//
// Reference: mq.c:85-127 (transfer_byte), :706-759 (mq_termination), :587-675
// (mq_truncation_length_min), tier1.c:2100-2130 (slope2log), :2161-2267
// (compute_convex_hull), :2477-2531 (distortion weights).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "device_common.cuh"
#include "t1_tables.cuh"

#define T1_HD __host__ __device__ __forceinline__

namespace bwcb {
namespace t1 {

using u64 = unsigned long long;

// ---- bit helpers ------------------------------------------------------------------------------
T1_HD int popc64(u64 x) {
#ifdef __CUDA_ARCH__
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}
T1_HD int ctz64(u64 x) {   // x != 0
#ifdef __CUDA_ARCH__
  return __ffsll((long long)x) - 1;
#else
  return __builtin_ctzll(x);
#endif
}
T1_HD int clz32(uint32_t x) {   // x != 0
#ifdef __CUDA_ARCH__
  return __clz((int)x);
#else
  return __builtin_clz(x);
#endif
}
T1_HD int bitlen_raw(bwc_raw q) {   // bits of q (0 for q == 0)
#ifdef __CUDA_ARCH__
  return q ? (int)(8 * sizeof(bwc_raw)) - (sizeof(bwc_raw) == 8 ? __clzll((long long)q) : __clz((int)(uint32_t)q)) : 0;
#else
  return q ? (int)(8 * sizeof(bwc_raw)) - (sizeof(bwc_raw) == 8 ? __builtin_clzll((unsigned long long)q)
                                                                 : __builtin_clz((unsigned)q)) : 0;
#endif
}

// ---- exactly rounded arithmetic (no contraction: device intrinsics, host IEEE operations built
// with -ffp-contract=off) -------------------------------------------------------------------------
T1_HD double mul_d(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
T1_HD double add_d(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
T1_HD double div_d(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
T1_HD bwc_float div_f(bwc_float a, bwc_float b) {
#ifdef __CUDA_ARCH__
  return dev::fdiv(a, b);
#else
  return a / b;
#endif
}
T1_HD bwc_raw raw_of(bwc_float f) {
#ifdef __CUDA_ARCH__
  return dev::as_raw(f);
#else
  bwc_raw r;
  std::memcpy(&r, &f, sizeof r);
  return r;
#endif
}
T1_HD bwc_float float_of(bwc_raw r) {
#ifdef __CUDA_ARCH__
  return dev::as_float(r);
#else
  bwc_float f;
  std::memcpy(&f, &r, sizeof f);
  return f;
#endif
}
// (bwc_raw)(|c| / step): quantisation of one coefficient, truncated toward zero
T1_HD bwc_raw quantise(bwc_float c_abs, bwc_float step) {
#ifdef __CUDA_ARCH__
  return dev::to_raw_rz(dev::fdiv(c_abs, step));
#else
  return (bwc_raw)(c_abs / step);
#endif
}
T1_HD double ll2d(long long v) {
#ifdef __CUDA_ARCH__
  return __ll2double_rn(v);
#else
  return (double)v;
#endif
}
T1_HD double ull2d(unsigned long long v) {
#ifdef __CUDA_ARCH__
  return __ull2double_rn(v);
#else
  return (double)v;
#endif
}
T1_HD uint64_t dbl_bits(double d) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t r;
  std::memcpy(&r, &d, sizeof r);
  return r;
#endif
}

// ---- MQ coder state and byte output ---------------------------------------------------------
struct MqState {
  uint32_t A, C, T;
  int32_t ct;   // shifts until the next byte transfer
  int32_t L;    // bytes emitted so far minus one (the first transfer emits nothing)
};

struct ByteSink {
  uint8_t *out;
  uint32_t cap;
  uint32_t flags;   // bit 0: output overflowed its capacity
};

// transfer_byte (mq.c:85-127), due now (ct == 0)
T1_HD void mq_transfer(MqState &e, ByteSink &bo) {
  if (e.T != 0xFF && (e.C & 0x8000000u)) {
    e.T++;
    e.C &= 0x7FFFFFFu;
  }
  if (e.L >= 0) {
    if ((uint32_t)e.L < bo.cap) bo.out[e.L] = (uint8_t)e.T; else bo.flags |= 1u;
  }
  e.L++;
  if (e.T == 0xFF) {
    e.T = (e.C >> 20) & 0xFF;
    e.C &= 0xFFFFFu;
    e.ct += 7;
  } else {
    e.T = (e.C >> 19) & 0xFF;
    e.C &= 0x7FFFFu;
    e.ct += 8;
  }
}

// mq_termination (mq.c:706-759)
T1_HD void mq_terminate(MqState &e, ByteSink &bo) {
  int n = 12 - e.ct;
  e.C <<= e.ct;
  e.ct = 0;
  while (n > 0) {
    mq_transfer(e, bo);
    n -= e.ct;
    e.C <<= e.ct;
    e.ct = 0;
  }
  mq_transfer(e, bo);
}

// end-of-pass coder state: A << 48 | T << 40 | ct << 32 | C, then L
T1_HD void mq_snapshot(const MqState &e, uint64_t *snaps, int p) {
  snaps[2 * p] = ((uint64_t)e.A << 48) | ((uint64_t)(e.T & 0xFF) << 40) |
                 ((uint64_t)(uint8_t)e.ct << 32) | (uint64_t)(uint32_t)e.C;
  snaps[2 * p + 1] = (uint64_t)(int64_t)e.L;
}

// Minimal number of bytes that decode a pass correctly, from the coder state at its end and the
// bytes emitted later (mq.c:587-675; the single-precision build uses 32-bit split arithmetic).
// Bytes at or beyond `cap` read as zero (the reference's buffer is zero-filled past its data).
T1_HD int64_t truncation_length(uint32_t A, uint32_t C, int32_t t, uint32_t T, int64_t L,
                                const uint8_t *p, uint32_t cap, uint32_t *bad) {
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
    const int32_t buff = (L >= 0 && L < (int64_t)cap) ? (int32_t)p[L] : 0;
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
    const int64_t buff = (L >= 0 && L < (int64_t)cap) ? (int64_t)p[L] : 0;
    L++;
    Cr -= buff << (35 - s);
    CAr -= buff << (35 - s);
    Cr = (int64_t)((uint64_t)Cr << s);
    CAr = (int64_t)((uint64_t)CAr << s);
    s = (buff == 0xFF) ? 7 : 8;
  }
#endif
  auto b = [&](int64_t i) -> uint32_t { return (i >= 0 && i < (int64_t)cap) ? p[i] : 0u; };
  if (L > 0 && b(L - 1) == 0xFF) L--;
  while (L > 1 && b(L - 2) == 0xFF && b(L - 1) == 0x7F) L -= 2;
  return L;
}

T1_HD uint16_t slope2log(double lambda) {
  const uint64_t raw = dbl_bits(lambda);
  const uint64_t exponent = ((raw & 0x7FF0000000000000ull) >> 44) - 0x41F00ull;
  const uint64_t mantissa = (raw & 0x000FFFFFFFFFFFFFull) >> 44;
#ifdef __CUDA_ARCH__
  const uint64_t r = (exponent + dev::c_frac2log[mantissa]) + 0x10000ull;
#else
  const uint64_t r = (exponent + dev::h_frac2log[mantissa]) + 0x10000ull;
#endif
  if (r > 0xFFFF) return 0xFFFF;
  if (r < 2) return 2;
  return (uint16_t)r;
}

// Everything after the MQ coding of one codeblock: termination, the zeroed margin after the
// codeword, per-pass truncation lengths, the convex hull of (length, distortion) and the 16-bit
// log slopes.  `snaps` holds the Z end-of-pass coder states and is reused as scratch for the
// hull; `dmse` the per-pass distortion decreases in the reference's integer units.  Returns the
// slope range (min over non-zero slopes << 16 | max) through *smin / *smax and or's problems
// into bo.flags: 2 hull stack underflow (the reference would read below its stack), 4 an
// unsettled truncation-length scan.
T1_HD void t1_finish(MqState &e, ByteSink &bo, int K, int Z, uint64_t *snaps,
                     const int64_t *dmse, double gain_step2, uint32_t *Lout, uint16_t *S,
                     uint32_t *smin_out, uint32_t *smax_out) {
  mq_terminate(e, bo);
  for (int i = 0; i < 16; ++i) {
    const int64_t q = (int64_t)e.L + i;
    if (q >= 0 && (uint64_t)q < bo.cap) bo.out[q] = 0;
  }
  uint32_t bad = 0;
  for (int j = 0; j < Z; ++j) {
    const uint64_t s0 = snaps[2 * j];
    const int64_t Ls = (int64_t)snaps[2 * j + 1];
    Lout[j] = (uint32_t)truncation_length((uint32_t)(s0 >> 48), (uint32_t)s0,
                                          (int32_t)(int8_t)((s0 >> 32) & 0xFF),
                                          (uint32_t)((s0 >> 40) & 0xFF), Ls, bo.out, bo.cap, &bad);
  }
  if (bad) bo.flags |= 4u;
  // hull scratch: slopes and the hull stack overwrite the snapshots
  double *lambda = reinterpret_cast<double *>(snaps);
  uint8_t *hull = reinterpret_cast<uint8_t *>(snaps + kMaxPasses + 1);
  double scale0 = gain_step2;
  scale0 = mul_d(scale0, ldexp(1.0, 2 * K));
  scale0 = div_d(scale0, 65536.0);
  // distortion decrease of pass q in the reference's weighting: the weight is scale0 for the
  // first plane and a quarter less per plane below (exact: powers of two, no subnormals); pass 0
  // codes plane K-1, passes 1-3 plane K-2, and so on
  auto mse_of = [&](int q) -> double {
    return mul_d(ll2d((long long)dmse[q]), ldexp(scale0, -2 * ((q + 2) / 3)));
  };
  for (int i = 0; i <= Z; ++i) lambda[i] = 0.0;
  for (int i = 0; i < Z; ++i) hull[i] = 0;
  lambda[0] = 18446744073709551616.0;
  int h = 0, hlast = 0;
  for (int i = 0; i < Z; ++i) {
    double dD = 0.0;
    for (int q = hlast; q <= i; ++q) dD = add_d(dD, mse_of(q));
    uint64_t dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
    if (dD > 0) {
      while (dD >= mul_d(lambda[hlast], ull2d(dL))) {
        lambda[hlast] = 0;
        if (h == 0) {
          bo.flags |= 2u;
          break;
        }
        h--;
        hlast = hull[h];
        dD = 0.0;
        for (int q = hlast; q <= i; ++q) dD = add_d(dD, mse_of(q));
        dL = (hlast > 0) ? (uint64_t)Lout[i] - Lout[hlast - 1] : (uint64_t)Lout[i];
      }
      h++;
      hlast = i + 1;
      hull[h] = (uint8_t)hlast;
      if (dL == 0)
        lambda[hlast] = (dD < 0) ? -1.0 : (dD == 0 ? 0.0 : 18446744073709551616.0);
      else
        lambda[hlast] = div_d(dD, ull2d(dL));
    } else {
      lambda[i + 1] = 0;
    }
  }
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
      smin = smin < v ? smin : v;
      smax = smax > v ? smax : v;
    }
  }
  *smin_out = smin;
  *smax_out = (Lout[Z - 1] > 0) ? smax : 0u;
  if (Lout[Z - 1] == 0) *smin_out = 0xFFFF;
}

// Upper bound of a codeblock's symbol stream in bytes at K bit planes: per bit plane a stripe
// column codes at most 6 decisions besides signs (run mode: run bit, two position bits, three
// samples below the first significant one), each sample one sign in its lifetime, 4
// segmentation symbols per plane, and every pass is padded to 16 bytes.
T1_HD uint64_t stream_bound(uint64_t ncols, uint32_t K) {
  return (ncols * (6ull * K + 4) + 4ull * K + 16ull * (3ull * K) + 31) & ~15ull;
}

}  // namespace t1
}  // namespace bwcb
