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

// One decision of the MQ coder (mq_bit_encode, mq.c:478-556), written as straight-line code:
// every branch of the reference's coder is a select, the context's new state is stored under a
// predicate, and the byte transfer that falls due during the renormalising shift (at most one in
// all but the rarest cases) is computed unconditionally and kept under a predicate.  Only a
// renormalisation long enough to need a second transfer (an interval of at most 0xFF, i.e. a
// less probable symbol in one of the most skewed states) takes a branch.
//   ent: the entry of the decision's context; on return the entry of the next decision's
//        context: nk == k and the state moved ? the new entry : nent (read before this decision)
T1_HD void mq_code_one(MqState &e, ByteSink &bo, uint32_t sym, uint32_t &ent, uint32_t nk,
                       uint32_t nent, uint32_t *slot, int stride, const uint32_t *tbl) {
  const uint32_t k = sym >> 1;
  const uint32_t em = tbl[(ent >> 17) & 0x7F], el = tbl[(ent >> 24) & 0x7F];
  const uint32_t qe = ent & 0xFFFFu;
  const uint32_t A1 = e.A - qe;
  const bool is_mps = ((sym ^ (ent >> 16)) & 1u) == 0u;
  const bool keep = is_mps != (A1 < qe);   // the interval keeps its upper part
  const uint32_t An = keep ? A1 : qe;
  e.C += keep ? qe : 0u;
  const bool ren = An < 0x8000u;
  const uint32_t ne = is_mps ? em : el;
  if (ren) slot[k * stride] = ne;
  ent = (ren && nk == k) ? ne : nent;
  const int sh = clz32(An) - 16;   // 0 without renormalisation
  e.A = An << sh;
  // shift up to the transfer point
  const int s1 = sh < e.ct ? sh : e.ct;
  e.C <<= s1;
  e.ct -= s1;
  const int rem = sh - s1;
  // transfer_byte (mq.c:85-127) when it fell due
  const bool tr = e.ct == 0;
  const uint32_t carry = (e.T != 0xFFu) ? ((e.C >> 27) & 1u) : 0u;
  const uint32_t T1 = e.T + carry;
  const uint32_t C1 = carry ? (e.C & 0x7FFFFFFu) : e.C;
  if (tr && (uint32_t)e.L < bo.cap) bo.out[e.L] = (uint8_t)T1;
  if (tr && e.L >= 0 && (uint32_t)e.L >= bo.cap) bo.flags |= 1u;
  const bool ff = T1 == 0xFFu;
  const uint32_t T2 = (C1 >> (ff ? 20 : 19)) & 0xFFu;
  const uint32_t C2 = C1 & (ff ? 0xFFFFFu : 0x7FFFFu);
  e.T = tr ? T2 : e.T;
  e.C = tr ? C2 : e.C;
  e.ct = tr ? (ff ? 7 : 8) : e.ct;
  e.L += tr ? 1 : 0;
  if (rem < e.ct) {
    e.C <<= rem;
    e.ct -= rem;
  } else {
    int r = rem;
    do {   // further transfers fall due: shift up to each, transfer, continue
      const int s2 = r < e.ct ? r : e.ct;
      e.C <<= s2;
      e.ct -= s2;
      r -= s2;
      if (e.ct == 0) mq_transfer(e, bo);
    } while (r > 0);
  }
}

T1_HD uint32_t chunk_sym(const Chunk &c, int j) { return (c.w[j >> 2] >> (8 * (j & 3))) & 0xFFu; }

// Codes Z passes of the stream at `src` (pcount[p] decisions in pass p), records the coder state
// at every pass end in snaps, and leaves the coder unterminated in `e`.  `slot` holds the 19
// context slots at a stride of `stride` words, `tbl` the 94-entry state table.  The stream must
// be readable 32 bytes past its end.  Full chunks of 16 decisions are coded without guards, so
// that consecutive decisions' independent work overlaps; a pass's last, partial chunk is coded
// decision by decision.
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
    // chunks follow each other through the passes (a pass's last chunk is padded), so the
    // stream is fetched in order, two chunks ahead
    const Chunk c = cur;
    cur = nxt;
    nxt = load_chunk(fetch);
    fetch += 16;
    uint32_t ent = slot[(chunk_sym(c, 0) >> 1) * stride];
    if (left >= 16u) {
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const uint32_t sym = chunk_sym(c, jj);
        const uint32_t nk = (jj < 15) ? (chunk_sym(c, jj + 1) >> 1) : 0xFFu;
        const uint32_t nent = (jj < 15) ? slot[nk * stride] : 0u;
        mq_code_one(e, bo, sym, ent, nk, nent, slot, stride, tbl);
      }
      left -= 16u;
    } else {
      for (uint32_t jj = 0; jj < left; ++jj) {
        const uint32_t sym = (c.w[jj >> 2] >> (8 * (jj & 3))) & 0xFFu;
        uint32_t nk = 0xFFu, nent = 0u;
        if (jj + 1 < left) {
          nk = ((c.w[(jj + 1) >> 2] >> (8 * ((jj + 1) & 3))) & 0xFFu) >> 1;
          nent = slot[nk * stride];
        }
        mq_code_one(e, bo, sym, ent, nk, nent, slot, stride, tbl);
      }
      left = 0;
    }
  }
}

// ---- the coder in two halves ------------------------------------------------------------------
// The coder's state splits into the interval A with the context states, which every decision
// needs from the one before it, and the code register C with its shift counter and byte output,
// which only consume, per decision, the value added to C (Qe when the interval keeps its upper
// part, else 0) and the renormalising shift.  The interval half (the producer) turns each chunk
// of decisions into those (add | shift << 16) pairs and the register half (the consumer) applies
// them, so each half is a dependent chain about half as long as the whole coder's.  Both walk
// the passes and chunks the same way, so each records its part of the coder state at every
// pass end; mq_code_stream's result is their combination, bit for bit.

// position in a codeblock's stream: pass p, decisions left in it, the next pass's count
struct MqWalk {
  const uint32_t *pcount;
  int Z, p;
  uint32_t left, next_count;
};

T1_HD void walk_init(MqWalk &w, const uint32_t *pcount, int Z) {
  w.pcount = pcount;
  w.Z = Z;
  w.p = 0;
  w.left = (Z > 0) ? pcount[0] : 0u;
  w.next_count = (Z > 1) ? pcount[1] : 0u;
}

T1_HD void walk_next_pass(MqWalk &w) {
  ++w.p;
  w.left = w.next_count;
  w.next_count = (w.p + 1 < w.Z) ? w.pcount[w.p + 1] : 0u;
}

// chunks of 16 decisions a stream is coded in (a pass's last chunk may be partial)
T1_HD uint32_t stream_chunks(const uint32_t *pcount, int Z) {
  uint32_t n = 0;
  for (int p = 0; p < Z; ++p) n += (pcount[p] + 15u) >> 4;
  return n;
}

// A context slot of the interval half: the context's state entry and the entries of its two
// successor states (after a more and a less probable symbol), so that a decision's next state
// is a select, not a table read; the successors of a new state are read from the table once,
// when the state is stored, a decision before they can be needed.
struct MqSlot {
  uint32_t cur, mps, lps, pad;
};

T1_HD MqSlot mq_slot_of(uint32_t ent, const uint32_t *tbl) {
  return MqSlot{ent, tbl[(ent >> 17) & 0x7F], tbl[(ent >> 24) & 0x7F], 0u};
}

// The interval half of mq_code_one: A and the context states; returns the decision's pair.
//   ent: the slot of the decision's context; on return the slot of the next decision's context
//   (nk == k and the state moved ? the new slot : nent, read before this decision)
T1_HD uint32_t mq_interval_one(uint32_t &A, uint32_t sym, MqSlot &ent, uint32_t nk,
                               const MqSlot &nent, MqSlot *slot, int stride,
                               const uint32_t *tbl) {
  const uint32_t k = sym >> 1;
  const uint32_t qe = ent.cur & 0xFFFFu;
  const uint32_t A1 = A - qe;
  const bool is_mps = ((sym ^ (ent.cur >> 16)) & 1u) == 0u;
  const bool keep = is_mps != (A1 < qe);
  const uint32_t An = keep ? A1 : qe;
  const bool ren = An < 0x8000u;
  const MqSlot ns = mq_slot_of(is_mps ? ent.mps : ent.lps, tbl);
  if (ren) slot[k * stride] = ns;
  const bool fwd = ren && nk == k;
  ent.cur = fwd ? ns.cur : nent.cur;
  ent.mps = fwd ? ns.mps : nent.mps;
  ent.lps = fwd ? ns.lps : nent.lps;
  const int sh = clz32(An) - 16;
  A = An << sh;
  return (keep ? qe : 0u) | ((uint32_t)sh << 16);
}

// The register half of mq_code_one: C, the shift counter and the byte transfers.  A transfer
// whose byte falls at or beyond the capacity is not stored; mq_consumer_passes' caller raises
// the overflow flag from the final byte count instead of per decision (the count only grows).
T1_HD void mq_register_one(MqState &e, ByteSink &bo, uint32_t pair) {
  const int sh = (int)(pair >> 16);
  e.C += pair & 0xFFFFu;
  const int s1 = sh < e.ct ? sh : e.ct;
  e.C <<= s1;
  e.ct -= s1;
  const int rem = sh - s1;
  const bool tr = e.ct == 0;
  const uint32_t carry = (e.T != 0xFFu) ? ((e.C >> 27) & 1u) : 0u;
  const uint32_t T1 = e.T + carry;
  const uint32_t C1 = carry ? (e.C & 0x7FFFFFFu) : e.C;
  if (tr && (uint32_t)e.L < bo.cap) bo.out[e.L] = (uint8_t)T1;
  const bool ff = T1 == 0xFFu;
  const uint32_t T2 = (C1 >> (ff ? 20 : 19)) & 0xFFu;
  const uint32_t C2 = C1 & (ff ? 0xFFFFFu : 0x7FFFFu);
  e.T = tr ? T2 : e.T;
  e.C = tr ? C2 : e.C;
  e.ct = tr ? (ff ? 7 : 8) : e.ct;
  e.L += tr ? 1 : 0;
  if (rem < e.ct) {
    e.C <<= rem;
    e.ct -= rem;
  } else {
    int r = rem;
    do {
      const int s2 = r < e.ct ? r : e.ct;
      e.C <<= s2;
      e.ct -= s2;
      r -= s2;
      if (e.ct == 0) mq_transfer(e, bo);
    } while (r > 0);
  }
}

struct MqProducer {
  MqWalk w;
  uint32_t A;
  const uint8_t *fetch;
  Chunk cur, nxt;
  MqSlot *slot;   // 19 context slots at `stride` slots
  int stride;
  const uint32_t *tbl;
};

T1_HD void mq_producer_init(MqProducer &P, const uint8_t *src, const uint32_t *pcount, int Z,
                            const uint32_t *tbl, MqSlot *slot, int stride) {
  for (int k = 0; k < dev::kCtxTotal; ++k)
    slot[k * stride] = mq_slot_of(tbl[dev::mq_initial_state(k)], tbl);
  walk_init(P.w, pcount, Z);
  P.A = 0x8000u;
  P.cur = load_chunk(src);
  P.nxt = load_chunk(src + 16);
  P.fetch = src + 32;
  P.slot = slot;
  P.stride = stride;
  P.tbl = tbl;
}

// Passes that end before the next chunk (empty ones too): A into snapA[p * sstride].
T1_HD void mq_producer_passes(MqProducer &P, uint16_t *snapA, int sstride) {
  while (P.w.p < P.w.Z && P.w.left == 0) {
    snapA[P.w.p * sstride] = (uint16_t)P.A;
    walk_next_pass(P.w);
  }
}

// Codes the next chunk into pairs[j * pstride]; returns its decision count, 0 at the end.
T1_HD uint32_t mq_produce_chunk(MqProducer &P, uint32_t *pairs, int pstride, uint16_t *snapA,
                                int sstride) {
  mq_producer_passes(P, snapA, sstride);
  if (P.w.p >= P.w.Z) return 0u;
  const Chunk c = P.cur;
  P.cur = P.nxt;
  P.nxt = load_chunk(P.fetch);
  P.fetch += 16;
  MqSlot *slot = P.slot;
  const int stride = P.stride;
  MqSlot ent = slot[(chunk_sym(c, 0) >> 1) * stride];
  if (P.w.left >= 16u) {
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const uint32_t sym = chunk_sym(c, jj);
      const uint32_t nk = (jj < 15) ? (chunk_sym(c, jj + 1) >> 1) : 0xFFu;
      const MqSlot nent = (jj < 15) ? slot[nk * stride] : MqSlot{0u, 0u, 0u, 0u};
      pairs[jj * pstride] = mq_interval_one(P.A, sym, ent, nk, nent, slot, stride, P.tbl);
    }
    P.w.left -= 16u;
    return 16u;
  }
  const uint32_t n = P.w.left;
  for (uint32_t jj = 0; jj < n; ++jj) {
    const uint32_t sym = (c.w[jj >> 2] >> (8 * (jj & 3))) & 0xFFu;
    uint32_t nk = 0xFFu;
    MqSlot nent{0u, 0u, 0u, 0u};
    if (jj + 1 < n) {
      nk = ((c.w[(jj + 1) >> 2] >> (8 * ((jj + 1) & 3))) & 0xFFu) >> 1;
      nent = slot[nk * stride];
    }
    pairs[jj * pstride] = mq_interval_one(P.A, sym, ent, nk, nent, slot, stride, P.tbl);
  }
  P.w.left = 0u;
  return n;
}

struct MqConsumer {
  MqWalk w;
  MqState e;
  ByteSink bo;
};

T1_HD void mq_consumer_init(MqConsumer &Q, const uint32_t *pcount, int Z, uint8_t *out,
                            uint32_t cap) {
  walk_init(Q.w, pcount, Z);
  Q.e = MqState{0x8000u, 0u, 0u, 12, -1};
  Q.bo = ByteSink{out, cap, 0u};
}

// The overflow flag of the transfers so far: some byte fell at or beyond the capacity exactly
// when the byte count passed it (a transfer that finds L >= 0 counts one byte).
T1_HD void mq_consumer_overflow(MqConsumer &Q) {
  if (Q.e.L > 0 && (uint32_t)Q.e.L > Q.bo.cap) Q.bo.flags |= 1u;
}

// Passes that end before the next chunk: the register part of the coder state into snaps (A
// is left zero there, for the interval half's value to be added).
T1_HD void mq_consumer_passes(MqConsumer &Q, uint64_t *snaps) {
  while (Q.w.p < Q.w.Z && Q.w.left == 0) {
    const MqState &e = Q.e;
    snaps[2 * Q.w.p] = ((uint64_t)(e.T & 0xFF) << 40) | ((uint64_t)(uint8_t)e.ct << 32) |
                       (uint64_t)(uint32_t)e.C;
    snaps[2 * Q.w.p + 1] = (uint64_t)(int64_t)e.L;
    walk_next_pass(Q.w);
  }
}

// Applies the next chunk's pairs[j * pstride]; returns its decision count, 0 at the end.
T1_HD uint32_t mq_consume_chunk(MqConsumer &Q, const uint32_t *pairs, int pstride,
                                uint64_t *snaps) {
  mq_consumer_passes(Q, snaps);
  if (Q.w.p >= Q.w.Z) return 0u;
  const uint32_t n = Q.w.left < 16u ? Q.w.left : 16u;
  for (uint32_t jj = 0; jj < n; ++jj) mq_register_one(Q.e, Q.bo, pairs[jj * pstride]);
  Q.w.left -= n;
  return n;
}

}  // namespace t1
}  // namespace bwcb
