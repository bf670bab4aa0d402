// MQ coding of one codeblock's symbol stream by one lane (a thread of the MQ kernel, or the host
// build of the kernel bodies).
//
// Reference: mq_bit_encode (mq.c:478-556), transfer_byte (mq.c:85-127), the probability-state
// table (mq.c:197-291), initialize_mq_encoder (mq.c:328-378).
//
// Input: the codeblock's symbol stream as the context-modelling kernel writes it -- pass after
// pass, one byte per decision (context << 1 | decision), each pass starting on a 16-byte boundary
// right after the previous one -- and the decision count of every pass.  The lane reads the
// stream 16 bytes at a time, two chunks ahead of the one it codes.
//
// Per decision the coder is written without branches except for byte transfers: with Qe the
// context's probability estimate and A' = A - Qe, the interval keeps the upper part (C += Qe,
// A = A') exactly when the decision equals the more probable symbol XOR A' < Qe, and takes Qe
// otherwise; the interval needs renormalising exactly when the new A is below 0x8000, and then
// the context moves to its next state (more probable or less probable branch of the table, the
// sense switch folded into the table), A and C shift left by the leading-zero count, and a byte
// falls due when the shift reaches the transfer counter.  Context slots hold full table entries;
// the next decision's slot is read before the current one is stored back (and forwarded when
// both use the same context), and both possible next entries are read from the table while the
// current decision is coded.
#pragma once

#include "t1_common.cuh"

namespace bwcb {
namespace t1 {

struct Chunk {
  uint32_t w[4];
};

T1_HD Chunk load_chunk(const uint8_t *p) {
  Chunk c;
#ifdef __CUDA_ARCH__
  const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(p));
  c.w[0] = v.x;
  c.w[1] = v.y;
  c.w[2] = v.z;
  c.w[3] = v.w;
#else
  std::memcpy(c.w, p, 16);
#endif
  return c;
}

// Codes Z passes of the stream at `src` (pcount[p] decisions in pass p), records the coder state
// at every pass end in snaps, and leaves the coder unterminated in `e`.  `slot` holds the 19
// context slots at a stride of `stride` words, `tbl` the 94-entry state table.  The stream must
// be readable 32 bytes past its end.
T1_HD void mq_code_stream(MqState &e, ByteSink &bo, const uint8_t *src, const uint32_t *pcount,
                          int Z, const uint32_t *tbl, uint32_t *slot, int stride,
                          uint64_t *snaps) {
  for (int k = 0; k < dev::kCtxTotal; ++k) slot[k * stride] = tbl[dev::mq_initial_state(k)];
  int p = 0;
  uint32_t left = (Z > 0) ? pcount[0] : 0u;
  uint32_t next_count = (Z > 1) ? pcount[1] : 0u;
  Chunk cur = load_chunk(src), nxt = load_chunk(src + 16);
  const uint8_t *fetch = src + 32;
  while (p < Z) {
    if (left == 0) {
      // end of pass p (possibly an empty one)
      mq_snapshot(e, snaps, p);
      ++p;
      left = next_count;
      next_count = (p + 1 < Z) ? pcount[p + 1] : 0u;
      continue;
    }
    const uint32_t cnt = left < 16u ? left : 16u;
    // chunks follow each other through the passes (a pass's last chunk is padded), so the
    // stream is fetched in order, two chunks ahead
    const Chunk c = cur;
    cur = nxt;
    nxt = load_chunk(fetch);
    fetch += 16;
    uint32_t ent = slot[((c.w[0] & 0xFF) >> 1) * stride];
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      if ((uint32_t)jj < cnt) {
        const uint32_t sym = (c.w[jj >> 2] >> (8 * (jj & 3))) & 0xFFu;
        const uint32_t k = sym >> 1;
        uint32_t nk = 0xFFu, nent = 0u;
        if (jj < 15 && (uint32_t)(jj + 1) < cnt) {
          nk = ((c.w[(jj + 1) >> 2] >> (8 * ((jj + 1) & 3))) & 0xFFu) >> 1;
          nent = slot[nk * stride];
        }
        const uint32_t em = tbl[(ent >> 17) & 0x7F], el = tbl[(ent >> 24) & 0x7F];
        const uint32_t qe = ent & 0xFFFFu;
        const uint32_t A1 = e.A - qe;
        const bool mps = ((sym ^ (ent >> 16)) & 1u) == 0u;
        const bool keep = mps != (A1 < qe);
        const uint32_t An = keep ? A1 : qe;
        e.C += keep ? qe : 0u;
        if (An < 0x8000u) {
          const uint32_t ne = mps ? em : el;
          slot[k * stride] = ne;
          if (nk == k) nent = ne;
          int sh = clz32(An) - 16;
          e.A = An << sh;
          if (sh < e.ct) {
            e.C <<= sh;
            e.ct -= sh;
          } else {
            do {   // shift up to each due transfer, transfer, continue
              const int s1 = sh < e.ct ? sh : e.ct;
              e.C <<= s1;
              e.ct -= s1;
              sh -= s1;
              if (e.ct == 0) mq_transfer(e, bo);
            } while (sh > 0);
          }
        } else {
          e.A = An;
        }
        ent = nent;
      }
    }
    left -= cnt;
  }
}

}  // namespace t1
}  // namespace bwcb
