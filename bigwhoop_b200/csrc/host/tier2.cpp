// Tier-2: PCRD rate control, packet headers and packet parsing.
//
// Rate control is the reference's per-layer bisection over 16-bit log slopes
// (tier2.c:1115-1254): every probe truncates each codeblock at its last pass whose slope is at
// or above the threshold, sums the body bytes and estimates every packet header
// (tier2.c:896-1079, :434-711).  The probe results feed a trajectory-dependent search (exact
// exits on equality, the `tmp` fallback), so the same arithmetic -- including its quirks, such
// as adding L[0] for a codeblock whose previous layer stopped after one pass -- is kept here.
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "common.hpp"
#include "../kernels/kernels.hpp"

namespace bwcb {

// (uint16)log2(x) of the reference for positive integers; x == 0 gives 0 (log2(0) = -inf,
// which x86-64 converts to the integer-indefinite value whose low 16 bits are 0)
static inline uint16_t ilog2_u16(uint64_t x) {
  if (!x) return 0;
  return (uint16_t)(63 - __builtin_clzll(x));
}

template <class Writer>
static void encode_delta_z(Writer &bw, int dz) {
  if (dz == 1) {
    bw.emit(0);
  } else if (dz == 2) {
    bw.emit(1); bw.emit(0);
  } else if (dz < 6) {
    dz -= 3;
    bw.emit(1); bw.emit(1);
    bw.emit(dz & 2); bw.emit(dz & 1);
  } else if (dz < 37) {
    dz -= 6;
    for (int i = 0; i < 4; ++i) bw.emit(1);
    for (int b = 4; b >= 0; --b) bw.emit(dz & (1 << b));
  } else if (dz < 293) {
    dz -= 37;
    for (int i = 0; i < 9; ++i) bw.emit(1);
    for (int b = 7; b >= 0; --b) bw.emit(dz & (1 << b));
  }
}

static int decode_delta_z(BitReader &br) {
  if (!br.get_bit()) return 1;
  if (!br.get_bit()) return 2;
  int dz = br.get_bit() << 1;
  dz |= br.get_bit();
  if (dz < 3) return dz + 3;
  dz = 0;
  for (int b = 4; b >= 0; --b) dz |= br.get_bit() << b;
  if (dz < 31) return dz + 6;
  dz = 0;
  for (int b = 7; b >= 0; --b) dz |= br.get_bit() << b;
  return dz + 37;
}

template <class Writer>
static void encode_length(Writer &bw, Codeblock &cb, int q, uchar estimate) {
  int16_t *cp = cb.cp();
  const int16_t z_curr = cp[q] - 1, z_prev = cp[q - 1] - 1;
  uint16_t beta = (!estimate) ? cb.beta : cb.beta_est;
  uint16_t max_beta = beta;
  const uint32_t L = (uint32_t)(cb.enc.L[z_curr] - ((z_prev >= 0) ? cb.enc.L[z_prev] : 0));
  const uint16_t cp_bits = ilog2_u16((uint64_t)(z_curr - z_prev));
  int32_t L_bits = (int32_t)ilog2_u16(L) + 1 - cp_bits;
  max_beta = (max_beta < L_bits) ? (uint16_t)L_bits : max_beta;
  while (beta < max_beta) {
    bw.emit(1);
    beta++;
  }
  bw.emit(0);
  const int sh = beta + cp_bits - 1;
  int64_t bitv = (sh >= 0 && sh < 31) ? ((int64_t)1 << sh) : 0;
  while (bitv > 0) {
    bw.emit(L & (uint32_t)bitv);
    bitv >>= 1;
  }
  if (estimate == 0) {
    cb.beta = beta;
    cb.beta_est = beta;
  } else if (estimate == 1) {
    cb.beta_est = beta;
  }
}

extern thread_local bool t_rate_control_in_parallel_fields;

// ---- parallel host loops ----------------------------------------------------------------------
// Rate control and packet assembly split into independent parts: a subband's precinct at one
// packet position (a segment) touches only its own codeblocks and tag trees, and every total
// they feed is an integer sum.  So those loops run on a small persistent pool of host threads,
// with results identical to running them in order: the final layer evaluation and the final
// headers over segments (their header bits joined in order afterwards), the probe tables and
// the probes over pieces of a packet's codeblocks (a probe's per-codeblock work is independent;
// only its header bits are then counted in order).
//
// run(n, fn) calls fn(i) for every i in [0, n) on the pool's threads and the calling thread and
// returns when all are done.  One call at a time: a second concurrent caller, a caller on one of
// the batch driver's per-field threads (the fields already run in parallel there), or a caller
// in a process forked after the pool started runs its loop on its own thread.
class WorkPool {
 public:
  static WorkPool &instance() {
    static WorkPool pool;
    return pool;
  }
  size_t size() const { return workers_.size() + 1; }
  void run(size_t n, const std::function<void(size_t)> &fn) {
    std::unique_lock<std::mutex> busy(call_, std::defer_lock);
    if (n <= 1 || workers_.empty() || t_rate_control_in_parallel_fields || getpid() != pid_ ||
        !busy.try_lock()) {
      for (size_t i = 0; i < n; ++i) fn(i);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(m_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      pending_.store(workers_.size());
      gen_.store(gen_.load() + 1);
    }
    cv_.notify_all();
    drain();
    spin([&] { return pending_.load(std::memory_order_acquire) == 0; });
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_.load() == 0; });
    fn_ = nullptr;
  }

 private:
  WorkPool() : pid_(getpid()) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = std::min(16u, hw ? hw : 1u);
    for (unsigned i = 1; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~WorkPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_.store(true);
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }
  void drain() {
    for (size_t i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*fn_)(i);
  }
  // Rate control calls run() many times in a row with short gaps (one probe after another), so
  // a thread that waits first polls for up to kSpinMicros before it sleeps: waking a sleeping
  // thread costs tens of microseconds, more than a probe's share of work.
  static constexpr int kSpinMicros = 200;
  template <class Ready>
  static void spin(Ready &&ready) {
    const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(kSpinMicros);
    for (;;) {
      for (int i = 0; i < 64; ++i) {
        if (ready()) return;
#if defined(__x86_64__) || defined(__i386__)
        __builtin_ia32_pause();
#elif defined(__aarch64__)
        asm volatile("yield");
#endif
      }
      if (std::chrono::steady_clock::now() >= until) return;
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      spin([&] { return stop_.load(std::memory_order_acquire) ||
                        gen_.load(std::memory_order_acquire) != seen; });
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_.load() || gen_.load() != seen; });
        if (stop_.load()) return;
        seen = gen_.load();
      }
      drain();
      std::lock_guard<std::mutex> lk(m_);
      if (pending_.fetch_sub(1) == 1) done_.notify_one();
    }
  }
  const pid_t pid_;
  std::vector<std::thread> workers_;
  std::mutex call_, m_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)> *fn_ = nullptr;
  size_t n_ = 0;
  std::atomic<size_t> next_{0}, pending_{0};
  std::atomic<uint64_t> gen_{0};
  std::atomic<bool> stop_{false};
};

// every packet position of the tile, in the order the codestream and the reference visit them
struct PacketRef {
  Parameter *par;
  Resolution *res;
  uint32_t p;
  uint64_t cb_base;   // index of the parameter's first codeblock in tile order
};

static std::vector<PacketRef> packet_list(Tile &tile) {
  std::vector<PacketRef> v;
  uint64_t cb_base = 0;
  for (Parameter &par : tile.params) {
    for (Resolution &res : par.res)
      for (uint64_t p = 0; p < res.nprec; ++p) v.push_back({&par, &res, (uint32_t)p, cb_base});
    cb_base += par.codeblocks.size();
  }
  return v;
}

void host_parallel(size_t n, const std::function<void(size_t)> &fn) {
  WorkPool::instance().run(n, fn);
}

// fn(first, last) over contiguous chunks of [0, n), a few chunks per pool thread
static void for_chunks(size_t n, const std::function<void(size_t, size_t)> &fn) {
  const size_t chunks = std::min(n, WorkPool::instance().size() * 4);
  if (chunks <= 1) {
    if (n) fn(0, n);
    return;
  }
  WorkPool::instance().run(chunks, [&](size_t c) { fn(n * c / chunks, n * (c + 1) / chunks); });
}

using BodyPieces = std::vector<std::pair<uint64_t, uint32_t>>;

// What the precinct of subband m at packet position p adds to the header of layer q's packet
// (create_packet's codeblock loop, tier2.c:434-711, for one subband): its header bits, unstuffed,
// and its body, counted (est 1) or as pieces (est 0).  Each subband's precinct has tag trees of
// its own, so different subbands can be coded at the same time and their bits joined in order.
static void segment_bits(Parameter &par, Resolution &res, uint32_t p, uint8_t m, int q,
                         uchar est, RawBits &hdr, uint64_t &body, BodyPieces &pieces) {
  const Subband &sb = par.subbands[res.first_subband + m];
  Precinct &pr = par.precincts[sb.first_precinct + p];
  for (uint64_t k = 0; k < pr.ncb; ++k) {
    Codeblock &cb = par.codeblocks[pr.first_cb + k];
    int16_t *cp = cb.cp();
    const int dz = cp[q] - cp[q - 1];
    if (cp[q - 1] == 0) {
      tagtree_encode_bits(pr.incl, hdr, (uint32_t)(q + 1), k, est);
      if (cp[q])
        for (uint32_t kk = 1; kk <= cb.enc.Kmsbs + 1u; ++kk)
          tagtree_encode_bits(pr.msbs, hdr, kk, k, est);
    } else {
      hdr.emit(dz);
    }
    if (dz) {
      encode_delta_z(hdr, dz);
      encode_length(hdr, cb, q, est);
      if (est <= 1) {
        const uint32_t start = (cp[q - 1] == 0) ? 0 : (uint32_t)cb.enc.L[cp[q - 1] - 1];
        const uint32_t end = (cp[q] == 0) ? 0 : (uint32_t)cb.enc.L[cp[q] - 1];
        if (est == 1)
          body += (uint32_t)(end - start);
        else
          pieces.emplace_back(cb.data_off + start, (uint32_t)(end - start));
      }
    }
  }
}

// create_packet (tier2.c:434-711).  est: 0 final, 1 final-size estimate, 2 probe.
static int64_t create_packet(Parameter &par, Resolution &res, uint32_t p, int q, uchar est) {
  Packet &pk = res.packets[(uint64_t)q * res.nprec + p];
  if (pk.e) {
    BitWriter hdr;
    hdr.mem.reserve(64);
    if (!est) pk.pieces.clear();
    hdr.emit(1);
    RawBits seg;
    uint64_t body = 0;
    for (uint8_t m = 0; m < res.nsub; ++m) {
      seg.clear();
      segment_bits(par, res, p, m, q, est, seg, body, pk.pieces);
      hdr.append(seg);
    }
    if (est == 1) pk.body_size += body;
    hdr.flush();
    if (est) {
      if (est == 2) pk.e = 0;
      return (int64_t)hdr.mem.size();
    }
    pk.header = std::move(hdr.mem);
    pk.size = pk.body_size + pk.header.size();
    return (int64_t)pk.header.size();
  }
  if (est) {
    if (est == 2) pk.e = 0;
    return 1;
  }
  pk.size = 1;
  pk.header.assign(1, 0);
  return 1;
}

// create_quality_layer's codeblock loop (tier2.c:896-1079) for the precinct of subband m at the
// position of r: each codeblock's truncation point for layer q under `threshold`, the body bytes
// that adds, and (final call) the tag-tree values; `grows` when a codeblock gains passes
static int64_t truncate_segment(const bwc_gl_ctrl &c, const PacketRef &r, uint8_t m,
                                uint16_t threshold, int q, uchar est, bool &grows) {
  Parameter &par = *r.par;
  Resolution &res = *r.res;
  const Subband &sb = par.subbands[res.first_subband + m];
  Precinct &pr = par.precincts[sb.first_precinct + r.p];
  int64_t size = 0;
  for (uint64_t k = 0; k < pr.ncb; ++k) {
    Codeblock &cb = par.codeblocks[pr.first_cb + k];
    int16_t *cp = cb.cp();
    int16_t z;
    for (z = cb.enc.Z; z >= 0 && cb.enc.S[z] < threshold; --z) {
    }
    if (z < cp[q - 1]) {
      cp[q] = cp[q - 1];
      if (cp[q] == 1) size += (int64_t)cb.enc.L[0];
    } else {
      cp[q] = z;
      if (z > 0) {
        size += (int64_t)cb.enc.L[z - 1];
        if (z > 1 && (cp[q - 1] > 0)) size -= (int64_t)cb.enc.L[cp[q - 1] - 1];
      }
    }
    if (cp[q] > cp[q - 1]) grows = true;
    if (!est) {
      if (q == 0) tagtree_set(pr.msbs, k, cb.enc.Kmsbs);
      if (q + 1 == c.nLayers) {
        uint8_t l;
        for (l = 0; (l < c.nLayers) && (cb.cp()[l] == 0); ++l) {
        }
        tagtree_set(pr.incl, k, l);
      }
    }
  }
  return size;
}

// create_quality_layer (tier2.c:896-1079) for one packet: the truncation points of the packet's
// codeblocks (every subband's precinct at that position), then the packet's header; used by the
// probe cross-check (the final evaluation runs per segment)
static int64_t quality_layer_packet(const bwc_gl_ctrl &c, const PacketRef &r, uint16_t threshold,
                                    int q, uchar est) {
  Resolution &res = *r.res;
  int64_t size = 0;
  bool grows = false;
  for (uint8_t m = 0; m < res.nsub; ++m)
    size += truncate_segment(c, r, m, threshold, q, est, grows);
  if (grows) res.packets[(uint64_t)q * res.nprec + r.p].e = 1;
  const int64_t ph = create_packet(*r.par, res, r.p, q, est + 1);
  return (ph < 0) ? -1 : size + ph;
}

// The final passes work on segments: one subband's precinct at one packet position (its
// codeblocks and tag trees belong to no other segment), taken largest first.
struct Segment {
  uint32_t packet;   // index into the packet list
  uint8_t m;         // subband within the resolution
  uint64_t ncb;
};

// segments of every packet, in packet then subband order (first[i]: packet i's first segment),
// and the order to work on them
static std::vector<Segment> segment_list(const std::vector<PacketRef> &pks,
                                         std::vector<uint32_t> &first,
                                         std::vector<uint32_t> &order) {
  std::vector<Segment> segs;
  first.assign(pks.size() + 1, 0);
  for (uint32_t i = 0; i < (uint32_t)pks.size(); ++i) {
    first[i] = (uint32_t)segs.size();
    const PacketRef &r = pks[i];
    for (uint8_t m = 0; m < r.res->nsub; ++m) {
      const Subband &sb = r.par->subbands[r.res->first_subband + m];
      segs.push_back({i, m, r.par->precincts[sb.first_precinct + r.p].ncb});
    }
  }
  first[pks.size()] = (uint32_t)segs.size();
  order.resize(segs.size());
  for (uint32_t j = 0; j < (uint32_t)segs.size(); ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return segs[a].ncb > segs[b].ncb; });
  return segs;
}

static int64_t create_quality_layer(bwc_codec *codec, Tile &tile, uint16_t threshold, int q,
                                    uchar est) {
  const bwc_gl_ctrl &c = codec->control;
  const std::vector<PacketRef> pks = packet_list(tile);
  std::atomic<int64_t> size{0};
  std::atomic<bool> bad{false};
  for_chunks(pks.size(), [&](size_t first, size_t last) {
    int64_t part = 0;
    for (size_t i = first; i < last; ++i) {
      const int64_t v = quality_layer_packet(c, pks[i], threshold, q, est);
      if (v < 0) bad = true; else part += v;
    }
    size += part;
  });
  return bad ? -1 : size.load();
}

// ---- rate-control probes ------------------------------------------------------------------
// Within the bisection of one layer, probes differ only in where each codeblock is truncated:
// the tag trees, the previous layer's truncation points and the length-code states stay fixed
// (an estimating probe changes none of them).  So each codeblock's tag-tree bits are derived
// once per layer, its truncation point comes from a binary search over its right-to-left slope
// records, and a packet header's size is counted by stuffing its bits a chunk at a time.  The
// result equals create_quality_layer(..., est = 1) exactly (same sums, same header bytes).

namespace {

// byte count of a bit string written with BitWriter::emit and BitWriter::flush: bytes of 8
// bits, except that a byte after 0xFF holds 7 (its top bit is the stuffed 0); a string ending
// right after 0xFF still gets that next byte
struct StuffCounter {
  uint64_t acc = 0;   // pending bits (the low `nacc`)
  int nacc = 0;
  int w = 8;          // width of the byte being filled
  uint64_t bytes = 0;
  void put(uint64_t v, int n) {   // the n (<= 56) low bits of v, most significant first
    acc = (acc << n) | (v & ((1ull << n) - 1));
    nacc += n;
    // a byte can only be 0xFF where 8 ones run in a row: with no such run among the pending
    // bits, and full bytes being filled, every whole byte is an 8-bit one
    uint64_t run = acc & (acc << 1);
    run &= run << 2;
    run &= run << 4;
    if (w == 8 && (run & ((nacc >= 64) ? ~0ull : ((1ull << nacc) - 1))) == 0) {
      bytes += (uint64_t)(nacc >> 3);
      nacc &= 7;
      return;
    }
    while (nacc >= w) {
      nacc -= w;
      const uint32_t byte = (uint32_t)(acc >> nacc) & ((1u << w) - 1);
      bytes++;
      w = (w == 8 && byte == 0xFF) ? 7 : 8;
    }
  }
  void put_bits(const RawBits &rb, uint64_t off, uint64_t n) {
    while (n) {
      const uint64_t b = off & 63;
      uint64_t m = 64 - b;
      if (m > n) m = n;
      if (m > 56) m = 56;
      put((rb.words[off >> 6] << b) >> (64 - m), (int)m);
      off += m;
      n -= m;
    }
  }
  // The first n bits of rb, given `lead` (their leading one bits, at most 8) and `runs` (the
  // ascending starts p of every 8-bit all-ones run in them): the bytes are counted from one
  // possible 0xFF to the next instead of bit by bit.  A byte is w bits (8, or 7 after an 0xFF
  // byte); from a byte start S (negative while bits before rb are pending), the next 0xFF can
  // only be a run starting at S + 8k, so the bytes up to it are counted at once.
  void put_run(const RawBits &rb, uint8_t lead, const std::vector<uint32_t> &runs) {
    const int64_t n = (int64_t)rb.n;
    if (!n) return;
    int64_t S = -(int64_t)nacc;                       // start of the byte being filled
    const uint64_t pend = acc & ((1ull << nacc) - 1);   // its bits from before rb
    size_t ri = 0;
    for (;;) {
      if (w == 7) {
        if (S + 7 > n) break;   // the 7-bit byte is not complete within rb
        bytes++;
        S += 7;
        w = 8;
        continue;
      }
      // w == 8: the first 0xFF byte at or after S, if any
      int64_t ff = 0;
      bool has_ff = false;
      if (S < 0) {
        // the byte mixing pending bits and rb's first bits
        if (S + 8 <= n && pend == (1ull << (-S)) - 1 && (int64_t)lead >= 8 + S) {
          ff = S;
          has_ff = true;
        }
        else if (S + 8 > n) break;   // not complete within rb
        else {
          bytes++;
          S += 8;
          continue;
        }
      } else {
        // runs before S are passed for good; a run at S + 8k + r (r != 0) may start a byte
        // once a 7-bit byte has shifted the boundaries, so it is only skipped here
        while (ri < runs.size() && (int64_t)runs[ri] < S) ++ri;
        for (size_t j = ri; j < runs.size(); ++j)
          if ((((int64_t)runs[j] - S) & 7) == 0) {
            ff = runs[j];
            has_ff = true;
            break;
          }
      }
      if (!has_ff) {   // no 0xFF byte: every whole byte left counts at once
        const int64_t k = (n - S) >> 3;
        bytes += (uint64_t)k;
        S += 8 * k;
        break;
      }
      bytes += (uint64_t)((ff - S) >> 3) + 1;   // the bytes before it, and the 0xFF byte
      S = ff + 8;
      w = 7;
    }
    // the bits of the byte being filled, [S, n)
    const int rest = (int)(n - S);
    acc = (S >= 0) ? read_bits(rb, (uint64_t)S, rest)
                   : ((pend << n) | read_bits(rb, 0, (int)n));
    nacc = rest;
  }
  // k (< 64) bits of rb from bit `off`, most significant first
  static uint64_t read_bits(const RawBits &rb, uint64_t off, int k) {
    if (k <= 0) return 0;
    const uint64_t i = off >> 6, b = off & 63;
    uint64_t v = rb.words[i] << b;
    if (b + (uint64_t)k > 64) v |= rb.words[i + 1] >> (64 - b);
    return v >> (64 - k);
  }
  uint64_t finish() const { return bytes + ((nacc > 0 || w == 7) ? 1 : 0); }
};

// what a probe reads of a codeblock, kept together (the codeblocks' own records are large and
// scattered: reading them per probe is cache-miss bound)
struct ProbeCb {
  int16_t zprev;            // truncation point of the previous layer
  uint16_t beta_est;        // length-code state of the estimates
  uint32_t rec_off, rec_n;  // slope records
  uint32_t pool;            // bit pool holding its tag-tree bits
  uint64_t L0, Lprev;       // L[0] and L[zprev - 1] (0 where they do not exist)
  uint64_t incl_off, msbs_off;
  uint32_t incl_n, msbs_n;
};

struct ProbePacket {
  uint32_t first, count;
  uint32_t piece0, npieces;   // its pieces (runs of at most piece_cbs() codeblocks)
};

// a run of codeblocks of one packet, the unit of parallel work
struct ProbePiece {
  uint32_t packet, first, count;   // codeblocks [first, first + count) of pr.cbs
};
// codeblocks per piece: 256, or BWC_B200_T2_PIECE (tests set a tiny size so that small fields
// split their packets into many pieces too)
static uint32_t piece_cbs() {
  static const uint32_t n = [] {
    const char *e = getenv("BWC_B200_T2_PIECE");
    const long v = e ? strtol(e, nullptr, 10) : 0;
    return (uint32_t)((v > 0 && v <= (1 << 20)) ? v : 256);
  }();
  return n;
}

struct Probe {
  // right-to-left slope records of every codeblock: z in decreasing order with strictly
  // increasing S; max{z : S[z] >= t} is the first record whose S >= t
  std::vector<uint16_t> rec_s;
  std::vector<int16_t> rec_z;
  std::vector<uint64_t> rec_L;     // L[z - 1] of the record's z (0 for z = 0)
  std::vector<uint32_t> rec_off;   // per codeblock in tile order (parameters concatenated)
  std::vector<ProbeCb> cbs;
  std::vector<ProbePacket> packets;
  std::vector<ProbePiece> pieces;
  std::vector<RawBits> pools;   // tag-tree bits, one pool per piece
};

// Appends to a bit string, most significant bit first, through a 64-bit register: only whole
// words are stored until finish() stores the rest.
struct BitSink {
  RawBits &rb;
  uint64_t acc = 0;   // the pending bits (the low `nacc`; nothing above them)
  int nacc = 0;
  explicit BitSink(RawBits &r) : rb(r) { rb.clear(); }
  void put(uint64_t v, int n) {   // the n (<= 57) low bits of v; v has no bits above them
    if (nacc + n < 64) {
      acc = (acc << n) | v;
      nacc += n;
    } else {
      const int k = 64 - nacc;   // 7 <= k <= n: the bits of v that complete the word
      rb.words.push_back((acc << k) | (v >> (n - k)));
      nacc = n - k;
      acc = nacc ? (v & ((1ull << nacc) - 1)) : 0;
    }
    rb.n += (uint64_t)n;
  }
  void put_range(const RawBits &src, uint64_t off, uint64_t n) {
    while (n) {
      const uint64_t b = off & 63;
      uint64_t m = 64 - b;
      if (m > n) m = n;
      if (m > 56) m = 56;
      put((src.words[off >> 6] << b) >> (64 - m), (int)m);
      off += m;
      n -= m;
    }
  }
  void finish() {
    if (nacc) rb.words.push_back(acc << (64 - nacc));
    nacc = 0;
    acc = 0;
  }
};

void build_records(Tile &tile, Probe &pr) {
  std::vector<const Codeblock *> all;
  for (Parameter &par : tile.params)
    for (Codeblock &cb : par.codeblocks) all.push_back(&cb);
  // records of a codeblock: the passes z (from Z down to 0) whose S exceeds every later one's
  auto walk = [](const CodedBlock &e, auto &&emit) {
    int best = -1;
    for (int z = e.Z; z >= 0; --z)
      if ((int)e.S[z] > best) {
        best = e.S[z];
        emit(z);
      }
  };
  pr.rec_off.assign(all.size() + 1, 0);
  for_chunks(all.size(), [&](size_t first, size_t last) {
    for (size_t i = first; i < last; ++i) {
      uint32_t n = 0;
      walk(all[i]->enc, [&](int) { ++n; });
      pr.rec_off[i + 1] = n;
    }
  });
  for (size_t i = 0; i < all.size(); ++i) pr.rec_off[i + 1] += pr.rec_off[i];
  pr.rec_s.resize(pr.rec_off.back());
  pr.rec_z.resize(pr.rec_off.back());
  pr.rec_L.resize(pr.rec_off.back());
  for_chunks(all.size(), [&](size_t first, size_t last) {
    for (size_t i = first; i < last; ++i) {
      const CodedBlock &e = all[i]->enc;
      uint32_t k = pr.rec_off[i];
      walk(e, [&](int z) {
        pr.rec_s[k] = e.S[z];
        pr.rec_z[k] = (int16_t)z;
        pr.rec_L[k] = z > 0 ? e.L[z - 1] : 0;
        ++k;
      });
    }
  });
}

// per-layer tables in the order create_packet visits codeblocks: the packets' codeblocks are
// laid out first, then pieces of at most piece_cbs() codeblocks are filled in parallel, each
// with its own pool of tag-tree bits (tag-tree estimates only read the trees)
void build_layer(Tile &tile, int q, Probe &pr) {
  const std::vector<PacketRef> pks = packet_list(tile);
  pr.packets.clear();
  pr.pieces.clear();
  uint32_t ncb = 0;
  for (uint32_t i = 0; i < (uint32_t)pks.size(); ++i) {
    const PacketRef &r = pks[i];
    uint32_t count = 0;
    for (uint8_t m = 0; m < r.res->nsub; ++m) {
      const Subband &sb = r.par->subbands[r.res->first_subband + m];
      count += (uint32_t)r.par->precincts[sb.first_precinct + r.p].ncb;
    }
    ProbePacket pk{ncb, count, (uint32_t)pr.pieces.size(), 0};
    const uint32_t per = piece_cbs();
    for (uint32_t b = 0; b < count; b += per) {
      pr.pieces.push_back({i, ncb + b, std::min(per, count - b)});
      pk.npieces++;
    }
    pr.packets.push_back(pk);
    ncb += count;
  }
  pr.cbs.assign(ncb, ProbeCb{});
  pr.pools.resize(pr.pieces.size());
  WorkPool::instance().run(pr.pieces.size(), [&](size_t ip) {
    const ProbePiece &pc = pr.pieces[ip];
    const PacketRef &r = pks[pc.packet];
    Parameter &par = *r.par;
    Resolution &res = *r.res;
    RawBits &pool = pr.pools[ip];
    pool.clear();
    // codeblock positions [lo, hi) within the packet, walked subband by subband
    const uint32_t lo = pc.first - pr.packets[pc.packet].first, hi = lo + pc.count;
    uint32_t pos = 0;
    for (uint8_t m = 0; m < res.nsub && pos < hi; ++m) {
      const Subband &sb = par.subbands[res.first_subband + m];
      const Precinct &prc = par.precincts[sb.first_precinct + r.p];
      for (uint64_t k = 0; k < prc.ncb; ++k, ++pos) {
        if (pos < lo || pos >= hi) continue;
        const uint64_t ci = prc.first_cb + k;
        Codeblock &cb = par.codeblocks[ci];
        ProbeCb &e = pr.cbs[pr.packets[pc.packet].first + pos];
        e.zprev = cb.cp()[q - 1];
        e.beta_est = cb.beta_est;
        e.L0 = cb.enc.Z > 0 ? cb.enc.L[0] : 0;
        e.Lprev = e.zprev > 0 ? cb.enc.L[e.zprev - 1] : 0;
        e.rec_off = pr.rec_off[r.cb_base + ci];
        e.rec_n = pr.rec_off[r.cb_base + ci + 1] - e.rec_off;
        e.pool = (uint32_t)ip;
        if (e.zprev == 0) {
          e.incl_off = pool.n;
          tagtree_estimate(prc.incl, pool, (uint32_t)(q + 1), k);
          e.incl_n = (uint32_t)(pool.n - e.incl_off);
          e.msbs_off = pool.n;
          for (uint32_t kk = 1; kk <= cb.enc.Kmsbs + 1u; ++kk)
            tagtree_estimate(prc.msbs, pool, kk, k);
          e.msbs_n = (uint32_t)(pool.n - e.msbs_off);
        }
      }
    }
  });
}

// index (in the tables) of the codeblock's first record with S >= threshold, or ~0u: a
// branch-free binary search (the records' S increase strictly; the outcome of each step is
// data, not a predictable branch)
inline uint32_t truncation_record(const Probe &pr, const ProbeCb &e, uint16_t threshold) {
  const uint16_t *s = pr.rec_s.data() + e.rec_off;
  uint32_t n = e.rec_n, lo = 0;   // the answer lies in [lo, lo + n]
  while (n > 1) {
    const uint32_t half = n >> 1;
    lo = (s[lo + half - 1] < threshold) ? lo + half : lo;
    n -= half;
  }
  if (n == 1 && s[lo] < threshold) ++lo;
  return (lo < e.rec_n) ? e.rec_off + lo : ~0u;
}

// One piece under one threshold: the body bytes its codeblocks add, whether any is included
// further (the packet's `e`), and its codeblocks' header bits in order.
struct PieceResult {
  int64_t body = 0;
  bool e = false;
  RawBits hdr;
  uint8_t lead = 0;             // leading one bits of hdr, at most 8
  std::vector<uint32_t> runs;   // starts of the 8-bit all-ones runs in hdr, ascending
};

// leading one bits (at most 8) and the starts of the runs of eight 1 bits of a bit string (its
// bits past n are zero, so no run reaches them)
static void scan_runs(const RawBits &rb, uint8_t &lead_out, std::vector<uint32_t> &runs) {
  runs.clear();
  lead_out = 0;
  const uint64_t n = rb.n;
  if (!n) return;
  const uint64_t *w = rb.words.data();
  const size_t nw = rb.words.size();
  const uint64_t inv = ~w[0];
  const uint64_t lead = inv ? (uint64_t)__builtin_clzll(inv) : 64;
  lead_out = (uint8_t)std::min<uint64_t>(std::min<uint64_t>(lead, 8), n);
  for (size_t i = 0; i < nw; ++i) {
    const uint64_t x = w[i], y = (i + 1 < nw) ? w[i + 1] : 0;
    uint64_t v = x;   // bit 63 - j set: stream bits 64 i + j .. 64 i + j + 7 are all ones
    for (int t = 1; t < 8; ++t) v &= (x << t) | (y >> (64 - t));
    while (v) {
      const int j = __builtin_clzll(v);
      runs.push_back((uint32_t)(64ull * i + (uint64_t)j));
      v &= ~(1ull << (63 - j));
    }
  }
}

void probe_piece(const Probe &pr, uint16_t threshold, const ProbePiece &pc, PieceResult &out) {
  out.body = 0;
  out.e = false;
  BitSink hb(out.hdr);
  for (uint32_t i = pc.first; i < pc.first + pc.count; ++i) {
    const ProbeCb &c = pr.cbs[i];
    const uint32_t r = truncation_record(pr, c, threshold);
    const int16_t z = (r != ~0u) ? pr.rec_z[r] : (int16_t)-1;
    const uint64_t Lz = (r != ~0u) ? pr.rec_L[r] : 0;   // L[z - 1]
    int16_t cpq;
    if (z < c.zprev) {
      cpq = c.zprev;
      if (cpq == 1) out.body += (int64_t)c.L0;
    } else {
      cpq = z;
      if (z > 0) {
        out.body += (int64_t)Lz;
        if (z > 1 && c.zprev > 0) out.body -= (int64_t)c.Lprev;
      }
    }
    const int dz = cpq - c.zprev;
    if (dz > 0) out.e = true;
    if (c.zprev == 0) {
      hb.put_range(pr.pools[c.pool], c.incl_off, c.incl_n);
      if (cpq) hb.put_range(pr.pools[c.pool], c.msbs_off, c.msbs_n);
    } else {
      hb.put(dz ? 1 : 0, 1);
    }
    if (!dz) continue;
    // encode_delta_z
    if (dz == 1) hb.put(0, 1);
    else if (dz == 2) hb.put(2, 2);
    else if (dz < 6) hb.put(12u | (uint32_t)(dz - 3), 4);
    else if (dz < 37) hb.put((15u << 5) | (uint32_t)(dz - 6), 9);
    else if (dz < 293) hb.put((511u << 8) | (uint32_t)(dz - 37), 17);
    // encode_length with the estimate state
    // here cpq = z > zprev: L[cpq - 1] is the record's, L[zprev - 1] the previous layer's
    const int16_t z_curr = cpq - 1, z_prev = c.zprev - 1;
    const uint16_t beta = c.beta_est;
    uint16_t max_beta = beta;
    const uint32_t L = (uint32_t)(Lz - ((z_prev >= 0) ? c.Lprev : 0));
    const uint16_t cp_bits = ilog2_u16((uint64_t)(z_curr - z_prev));
    const int32_t L_bits = (int32_t)ilog2_u16(L) + 1 - cp_bits;
    max_beta = (max_beta < L_bits) ? (uint16_t)L_bits : max_beta;
    for (int n1 = max_beta - beta; n1 > 0; n1 -= 32) {
      const int m = n1 < 32 ? n1 : 32;
      hb.put((1ull << m) - 1, m);
    }
    hb.put(0, 1);
    const int sh = max_beta + cp_bits - 1;
    if (sh >= 0 && sh < 31) hb.put(L & (uint32_t)((2ull << sh) - 1), sh + 1);
  }
  hb.finish();
  scan_runs(out.hdr, out.lead, out.runs);
}

// create_quality_layer(codec, tile, threshold, q, 1) for the tables of layer q, for several
// thresholds at once: every (threshold, piece) pair is a task on the pool, then every
// threshold's packets are sized (a packet header: a 1 bit, its pieces' bits, byte stuffing;
// an empty packet: one byte) as a task of its own
void probe_thresholds(const Probe &pr, const std::vector<uint16_t> &thr, std::vector<int64_t> &out) {
  const size_t nt = thr.size(), np = pr.pieces.size();
  // result buffers of the calling thread, kept (with their capacity) from probe to probe; the
  // pool's tasks reach them through this reference (a thread_local named inside the tasks would
  // be each worker's own)
  thread_local std::vector<PieceResult> part_tls;
  std::vector<PieceResult> &part = part_tls;
  if (part.size() < nt * np) part.resize(nt * np);
  WorkPool::instance().run(nt * np, [&](size_t i) {
    probe_piece(pr, thr[i / np], pr.pieces[i % np], part[i]);
  });
  out.assign(nt, 0);
  WorkPool::instance().run(nt, [&](size_t k) {
    int64_t size = 0;
    for (const ProbePacket &pk : pr.packets) {
      StuffCounter sc;
      sc.put(1, 1);
      bool e = false;
      for (uint32_t j = pk.piece0; j < pk.piece0 + pk.npieces; ++j) {
        const PieceResult &r = part[k * np + j];
        size += r.body;
        e = e || r.e;
        sc.put_run(r.hdr, r.lead, r.runs);
      }
      size += e ? (int64_t)sc.finish() : 1;
    }
    out[k] = size;
  });
}

// create_quality_layer(codec, tile, threshold, q, 0) over segments in parallel: truncation
// points and tag-tree values of every segment; then the packets' `e`; then every segment's header
// bits (estimating: the trees are only read, the length codes' estimate state advances); then
// each packet's header is sized as a probe sizes it (a 1 bit, its segments' bits, byte stuffing;
// an empty packet: one byte).  Same sums, same states as the packet-at-a-time loop.
int64_t final_quality_layer(bwc_codec *codec, Tile &tile, uint16_t threshold, int q) {
  const bwc_gl_ctrl &c = codec->control;
  const std::vector<PacketRef> pks = packet_list(tile);
  std::vector<uint32_t> first, order;
  const std::vector<Segment> segs = segment_list(pks, first, order);
  const size_t ns = segs.size();
  std::vector<int64_t> size(ns, 0);
  std::vector<uint8_t> grows(ns, 0);
  WorkPool::instance().run(ns, [&](size_t j) {
    const uint32_t s = order[j];
    bool g = false;
    size[s] = truncate_segment(c, pks[segs[s].packet], segs[s].m, threshold, q, 0, g);
    grows[s] = g ? 1 : 0;
  });
  std::vector<uint8_t> e(pks.size(), 0);
  for (size_t i = 0; i < pks.size(); ++i) {
    Packet &pk = pks[i].res->packets[(uint64_t)q * pks[i].res->nprec + pks[i].p];
    for (uint32_t s = first[i]; s < first[i + 1]; ++s)
      if (grows[s]) pk.e = 1;
    e[i] = pk.e;
  }
  std::vector<RawBits> bits(ns);
  std::vector<uint64_t> body(ns, 0);
  std::vector<uint8_t> lead(ns, 0);
  std::vector<std::vector<uint32_t>> runs(ns);
  WorkPool::instance().run(ns, [&](size_t j) {
    const uint32_t s = order[j];
    if (!e[segs[s].packet]) return;
    const PacketRef &r = pks[segs[s].packet];
    BodyPieces unused;
    segment_bits(*r.par, *r.res, r.p, segs[s].m, q, 1, bits[s], body[s], unused);
    scan_runs(bits[s], lead[s], runs[s]);
  });
  int64_t total = 0;
  for (size_t i = 0; i < pks.size(); ++i) {
    for (uint32_t s = first[i]; s < first[i + 1]; ++s) total += size[s];
    if (!e[i]) {
      total += 1;
      continue;
    }
    Packet &pk = pks[i].res->packets[(uint64_t)q * pks[i].res->nprec + pks[i].p];
    StuffCounter sc;
    sc.put(1, 1);
    for (uint32_t s = first[i]; s < first[i + 1]; ++s) {
      sc.put_run(bits[s], lead[s], runs[s]);
      pk.body_size += body[s];
    }
    total += (int64_t)sc.finish();
  }
  return total;
}

}  // namespace

// ---- rate-control warm start ---------------------------------------------------------------
// The reference's per-layer bisection (tier2.c:1115-1254) is a chain of dependent probes, each
// a full truncation-and-header estimate.  Its outcome depends on the exact sequence of probes,
// so the search itself is kept: the same probes, compared the same way, in the same order.
// What a predicted final threshold changes is WHEN the probes are evaluated: from the
// prediction the probe path is simulated (assuming the size falls as the threshold rises) and
// its next few probes are evaluated at once, in parallel host threads; the exact bisection then
// replays over those results, and only when it leaves them is a new round needed (again
// speculated from the prediction).  The selected slope, and so every output byte, is the
// plain search's; what the prediction saves is rounds of dependent probes.
//
// Features of one layer (kRateFeatures values): a 32-bin histogram (fractions) of the
// codeblocks' non-zero pass slopes S[1..Z] over the 16-bit log range, log(bits per value of the
// layer) / 4 and (log(values) - 14) / 4.  The network predicts the final slope / 65536.

namespace {

// counts[i] = codeblock passes (z >= 1, non-zero slope) with S >> 11 == i; counts[32] = total
static void rate_histogram(const Tile &tile, uint64_t counts[33]) {
  std::vector<const Codeblock *> all;
  for (const Parameter &par : tile.params)
    for (const Codeblock &cb : par.codeblocks) all.push_back(&cb);
  std::mutex m;
  for (int i = 0; i < 33; ++i) counts[i] = 0;
  for_chunks(all.size(), [&](size_t first, size_t last) {
    uint64_t c[33] = {};
    for (size_t k = first; k < last; ++k) {
      const CodedBlock &enc = all[k]->enc;
      for (int z = 1; z <= enc.Z; ++z)
        if (enc.S[z]) {
          c[enc.S[z] >> 11]++;
          c[32]++;
        }
    }
    std::lock_guard<std::mutex> lk(m);
    for (int i = 0; i < 33; ++i) counts[i] += c[i];
  });
}

static void rate_features_from(const Tile &tile, const uint64_t counts[33], float bpv, float *out) {
  const double total = (double)counts[32];
  for (int i = 0; i < 32; ++i) out[i] = total > 0 ? (float)((double)counts[i] / total) : 0.f;
  uint64_t values = tile.box.size() * tile.params.size();
  out[32] = (float)(std::log((double)std::max(bpv, 1e-6f)) / 4.0);
  out[33] = (float)((std::log((double)std::max<uint64_t>(values, 1)) - 14.0) / 4.0);
}

void rate_features(const Tile &tile, float bpv, float *out) {
  uint64_t counts[33];
  rate_histogram(tile, counts);
  rate_features_from(tile, counts, bpv, out);
}

// One bisection step of tier2.c:1115-1254; returns true when the search is over.
struct Search {
  uint16_t smin, smax, tmp, slope;
  int64_t est;
  bool done() const { return smin >= smax; }
  uint16_t next() const { return (uint16_t)((smax + smin) >> 1); }
  void step(uint16_t s, int64_t e, int64_t target) {
    slope = s;
    est = e;
    if (e > target) {
      if (smin == s) smax = s;
      smin = s;
    } else if (e < target) {
      if (smax == s) smin = s;
      smax = s;
      tmp = s;
    } else {
      smax = s;
      smin = s;
    }
  }
};

// the probe slopes the search would take if its estimate exceeded the target exactly below
// `pred` (the predicted final slope)
std::vector<uint16_t> predicted_path(Search st, uint16_t pred, int64_t target) {
  std::vector<uint16_t> out;
  while (!st.done() && out.size() < 64) {
    const uint16_t s = st.next();
    out.push_back(s);
    st.step(s, (s < pred) ? target + 1 : target - 1, target);
  }
  return out;
}

}  // namespace

// Set by the batch driver in its worker threads: the fields already run in parallel there, so
// the speculative probes of one field are not spread over further threads.
thread_local bool t_rate_control_in_parallel_fields = false;

// probes of the predicted path evaluated per round (the first being the one the search needs)
constexpr size_t kSpeculatedProbes = 4;

// create_quality_layers (tier2.c:1115-1254)
static uchar create_quality_layers(bwc_codec *codec, Tile &tile) {
  const bwc_gl_ctrl &c = codec->control;
  const bwc_gl_inf &info = codec->info;
  int64_t est_tile = 0, target = 0, est = 0;
  const uint32_t main_header = (uint32_t)c.headerSize;
  const uint64_t tile_size = tile.box.size() * (uint64_t)info.nPar;
  const uint64_t header_size =
      (uint64_t)ceilf((float)(main_header + tile.header_size) / (float)c.nLayers);
  static const bool check = getenv("BWC_B200_CHECK_PROBES") != nullptr;
  Probe probe;
  build_records(tile, probe);
  // features and, when a model is set, the predicted final slope of every layer
  tile.rc_features.assign((size_t)c.nLayers * kRateFeatures, 0.f);
  tile.rc_stats.assign((size_t)c.nLayers * kRateStats, 0.0);
  uint64_t counts[33];
  rate_histogram(tile, counts);
  for (uint8_t l = 0; l < c.nLayers; ++l)
    rate_features_from(tile, counts, c.bitrate[l], tile.rc_features.data() + (size_t)l * kRateFeatures);
  std::vector<float> pred(c.nLayers, -1.f);
  const bool have_pred =
      !check && c.nLayers <= 64 && mlp_predict(tile.rc_features.data(), c.nLayers, pred.data());
  // with no spare threads the prediction is recorded but probes are evaluated on demand
  const bool speculate = have_pred && !t_rate_control_in_parallel_fields;
  for (uint8_t l = 0; l < c.nLayers; ++l) {
    uint16_t slope;
    int probes = 0, rounds = 0;
    uint16_t pslope = 0;
    target = (int64_t)ceilf(c.bitrate[l] * (float)tile_size / 8.0f);
    if ((float)target > 0.0f) {
      Search st{tile.slope_min, tile.slope_max, tile.slope_min, tile.slope_min, 0};
      build_layer(tile, l, probe);
      if (have_pred) {
        const double p = std::min(std::max((double)pred[l], 0.0), 1.0) * 65536.0;
        pslope = (uint16_t)std::min(65535.0, std::floor(p));
      }
      std::vector<std::pair<uint16_t, int64_t>> known;   // evaluated probes of this layer
      auto lookup = [&](uint16_t s, int64_t *e) {
        for (auto &kv : known)
          if (kv.first == s) {
            *e = kv.second;
            return true;
          }
        return false;
      };
      while (!st.done()) {
        const uint16_t s = st.next();
        int64_t e;
        if (!lookup(s, &e)) {
          // a new round: this probe, plus the rest of the predicted path
          std::vector<uint16_t> todo{s};
          if (speculate) {
            todo = predicted_path(st, pslope, target - est_tile - (int64_t)header_size);
            if (todo.empty() || todo[0] != s) todo.insert(todo.begin(), s);
            // the next few probes of the path: deeper ones are rarely reached before the
            // search leaves the path, and each costs a full probe
            if (todo.size() > kSpeculatedProbes) todo.resize(kSpeculatedProbes);
          }
          std::vector<int64_t> res;
          probe_thresholds(probe, todo, res);
          for (size_t k = 0; k < todo.size(); ++k) known.emplace_back(todo[k], res[k]);
          ++rounds;
          e = res[0];
        }
        if (check) {
          const int64_t slow = create_quality_layer(codec, tile, s, l, 1);
          if (slow != e) {
            fprintf(stderr, "bwc: rate-control probe mismatch (layer %d, slope %u: %lld vs %lld)\n",
                    l, s, (long long)e, (long long)slow);
            return 1;
          }
        }
        if (e < 0) return 1;
        ++probes;
        st.step(s, e + est_tile + (int64_t)header_size, target);
      }
      slope = st.slope;
      est = st.est;
      if (probes == 0) slope = tile.slope_min;
      if (est > target && probes > 0) slope = std::max(st.tmp, tile.slope_min);
    } else {
      slope = 0;
    }
    double *rs = tile.rc_stats.data() + (size_t)l * kRateStats;
    rs[0] = slope;
    rs[1] = probes;
    rs[2] = rounds;
    rs[3] = have_pred ? (double)pslope : -1.0;
    rs[4] = tile.slope_min;
    rs[5] = tile.slope_max;
    est = final_quality_layer(codec, tile, slope, l);
    if (est >= 0)
      est_tile += est + (int64_t)header_size;
    else
      return 1;
  }
  return 0;
}

// create_packets (tier2.c:751-849): final headers for every packet, then the per-codeblock
// coding state is cleared as in the reference.  Each segment codes its layers in order (its tag
// trees and length codes carry state from layer to layer) in parallel with the others; then
// every packet's header is its segments' bits joined in subband order behind the leading 1 bit.
static uchar create_packets(bwc_codec *codec, Tile &tile) {
  const bwc_gl_ctrl &c = codec->control;
  const int nl = c.nLayers;
  const std::vector<PacketRef> pks = packet_list(tile);
  std::vector<uint32_t> first, order;
  const std::vector<Segment> segs = segment_list(pks, first, order);
  std::vector<RawBits> bits(segs.size() * (size_t)nl);
  std::vector<BodyPieces> body(segs.size() * (size_t)nl);
  WorkPool::instance().run(segs.size(), [&](size_t j) {
    const uint32_t s = order[j];
    const PacketRef &r = pks[segs[s].packet];
    Parameter &par = *r.par;
    Resolution &res = *r.res;
    uint64_t unused = 0;
    for (int l = 0; l < nl; ++l)
      if (res.packets[(uint64_t)l * res.nprec + r.p].e)
        segment_bits(par, res, r.p, segs[s].m, l, 0, bits[(size_t)s * nl + l], unused,
                     body[(size_t)s * nl + l]);
    // the reference clears each codeblock's coding state once its packets exist
    const Subband &sb = par.subbands[res.first_subband + segs[s].m];
    const Precinct &pr = par.precincts[sb.first_precinct + r.p];
    for (uint64_t k = 0; k < pr.ncb; ++k) {
      Codeblock &cb = par.codeblocks[pr.first_cb + k];
      cb.enc = CodedBlock();
      for (int l = 0; l < nl; ++l) cb.cp()[l] = 0;
    }
  });
  for_chunks(pks.size() * (size_t)nl, [&](size_t lo, size_t hi) {
    for (size_t x = lo; x < hi; ++x) {
      const size_t i = x / nl;
      const int l = (int)(x % nl);
      Packet &pk = pks[i].res->packets[(uint64_t)l * pks[i].res->nprec + pks[i].p];
      if (!pk.e) {
        pk.size = 1;
        pk.header.assign(1, 0);
        continue;
      }
      BitWriter hdr;
      hdr.emit(1);
      pk.pieces.clear();
      for (uint32_t s = first[i]; s < first[i + 1]; ++s) {
        hdr.append(bits[(size_t)s * nl + l]);
        const BodyPieces &b = body[(size_t)s * nl + l];
        pk.pieces.insert(pk.pieces.end(), b.begin(), b.end());
      }
      hdr.flush();
      pk.header = std::move(hdr.mem);
      pk.size = pk.body_size + pk.header.size();
    }
  });
  return 0;
}

uchar t2_encode(bwc_codec *codec, Tile &tile) {
  if (create_quality_layers(codec, tile)) return 1;
  if (create_packets(codec, tile)) return 1;
  return 0;
}

// false on a run of 1 bits longer than any length code needs: a corrupt or truncated header
// (past its end the reader yields 1 bits, so the loop would not end)
static bool decode_length(BitReader &br, Codeblock &cb, int q) {
  while (br.get_bit())
    if (++cb.beta > 64) return false;
  int16_t *cp = cb.cp();
  const int16_t z_curr = cp[q] - 1, z_prev = cp[q - 1] - 1;
  uint16_t L_bits = (uint16_t)(cb.beta + ilog2_u16((uint64_t)(z_curr - z_prev)));
  uint32_t i = 0;
  for (; L_bits > 0; --L_bits) {
    i <<= 1;
    i |= br.get_bit();
  }
  cb.enc.L[z_curr] = ((z_prev >= 0) ? cb.enc.L[z_prev] : 0) + i;
  return true;
}

// parse_packet (tier2.c:1364-1684).  `pos` is the packet's first byte in the codestream,
// `body_size` the tile body bytes still unread.  The body is taken to start where the bit
// reader stopped (its byte index, not bytes_used), as in the reference.
uchar parse_packet(bwc_codec *codec, Tile &tile, Packet &pk, const uint8_t *cs, uint64_t cs_len,
                   uint64_t pos, uint64_t body_size) {
  Parameter &par = tile.params[pk.c];
  Resolution &res = par.res[pk.r];
  const int q = pk.l;
  BitReader br;
  br.mem = cs + pos;
  br.Lmax = (uint32_t)body_size;
  if (pos + br.Lmax > cs_len) br.Lmax = cs_len - pos;
  pk.e = br.get_bit();
  for (uint8_t m = 0; m < res.nsub; ++m) {
    const Subband &sb = par.subbands[res.first_subband + m];
    Precinct &pr = par.precincts[sb.first_precinct + pk.p];
    for (uint64_t k = 0; k < pr.ncb; ++k) {
      Codeblock &cb = par.codeblocks[pr.first_cb + k];
      int16_t *cp = cb.cp();
      if (pk.e) {
        int dz = 0;
        if (cp[q - 1] == 0) {
          tagtree_decode(pr.incl, br, (uint32_t)(q + 1), k);
          if (pr.incl.nodes[k].value <= q) {
            dz = 1;
            // no bit-plane count reaches 255: beyond it the header is corrupt
            if (!tagtree_decode_until_known(pr.msbs, br, k, 255)) return 1;
            if (pr.msbs.nodes[k].value > sb.Kmax) return 1;   // more missing planes than exist
            cb.enc.Kmsbs = (uint8_t)pr.msbs.nodes[k].value;
          }
        } else {
          dz = br.get_bit();
        }
        cp[q] = cp[q - 1];
        if (dz) {
          dz = decode_delta_z(br);
          cp[q] += dz;
          // no more passes than the codeblock's bit planes have (3 K - 2): a corrupt header
          // would otherwise index past the pass tables here and in the decoder
          if (cp[q] > 3 * (int)(sb.Kmax - cb.enc.Kmsbs) - 2 || cp[q] > kMaxPasses) return 1;
          cb.enc.Z = (uint8_t)cp[q];
          if (!decode_length(br, cb, q)) return 1;
        }
      } else {
        cp[q] = cp[q - 1];
      }
    }
  }
  if (!pk.header_len) pk.header_len = br.bytes_used();
  pk.header_pos = pos;
  uint64_t body = pos + br.L;
  if (codec->control.error_resilience) {
    if (body + 2 > cs_len || cs[body] != 0xFF || cs[body + 1] != 0x92) return 1;
    body += 2;
    pk.header_len += 2;
  }
  pk.body_pos = body;
  pk.body_size = 0;
  if (pk.e) {
    uint64_t at = body;
    for (uint8_t m = 0; m < res.nsub; ++m) {
      const Subband &sb = par.subbands[res.first_subband + m];
      Precinct &pr = par.precincts[sb.first_precinct + pk.p];
      for (uint64_t k = 0; k < pr.ncb; ++k) {
        Codeblock &cb = par.codeblocks[pr.first_cb + k];
        int16_t *cp = cb.cp();
        if (cp[q] > cp[q - 1]) {
          const uint32_t start = (cp[q - 1] == 0) ? 0 : (uint32_t)cb.enc.L[cp[q - 1] - 1];
          const uint32_t end = (cp[q] == 0) ? 0 : (uint32_t)cb.enc.L[cp[q] - 1];
          const uint32_t size = end - start;
          if (at + size > cs_len) return 1;
          if (cb.chunks.empty()) cb.chunks.reserve(codec->control.nLayers);   // one allocation
          cb.chunks.emplace_back(at, size);
          at += size;
          pk.body_size += size;
        }
      }
    }
  }
  pk.size = pk.header_len + pk.body_size;
  return 0;
}

}  // namespace bwcb
