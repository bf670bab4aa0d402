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

static void encode_delta_z(BitWriter &bw, int dz) {
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

static void encode_length(BitWriter &bw, Codeblock &cb, int q, uchar estimate) {
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

// ---- packet-parallel host loops --------------------------------------------------------------
// Rate control and packet assembly work packet by packet: a packet's computations touch only its
// own codeblocks, its precincts' tag trees and the packet itself, and every total they feed is
// an integer sum.  So those loops run over chunks of packets on a small persistent pool of host
// threads, with results identical to running them in order.
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
      pending_ = workers_.size();
      ++gen_;
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
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
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }
  void drain() {
    for (size_t i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*fn_)(i);
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      drain();
      std::lock_guard<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  const pid_t pid_;
  std::vector<std::thread> workers_;
  std::mutex call_, m_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)> *fn_ = nullptr;
  size_t n_ = 0, pending_ = 0;
  std::atomic<size_t> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
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

// fn(first, last) over contiguous chunks of [0, n), a few chunks per pool thread
static void for_chunks(size_t n, const std::function<void(size_t, size_t)> &fn) {
  const size_t chunks = std::min(n, WorkPool::instance().size() * 4);
  if (chunks <= 1) {
    if (n) fn(0, n);
    return;
  }
  WorkPool::instance().run(chunks, [&](size_t c) { fn(n * c / chunks, n * (c + 1) / chunks); });
}

// create_packet (tier2.c:434-711).  est: 0 final, 1 final-size estimate, 2 probe.
static int64_t create_packet(Parameter &par, Resolution &res, uint32_t p, int q, uchar est) {
  Packet &pk = res.packets[(uint64_t)q * res.nprec + p];
  if (pk.e) {
    BitWriter hdr;
    hdr.mem.reserve(64);
    if (!est) pk.pieces.clear();
    hdr.emit(1);
    for (uint8_t m = 0; m < res.nsub; ++m) {
      const Subband &sb = par.subbands[res.first_subband + m];
      Precinct &pr = par.precincts[sb.first_precinct + p];
      for (uint64_t k = 0; k < pr.ncb; ++k) {
        Codeblock &cb = par.codeblocks[pr.first_cb + k];
        int16_t *cp = cb.cp();
        const int dz = cp[q] - cp[q - 1];
        if (cp[q - 1] == 0) {
          tagtree_encode(pr.incl, hdr, (uint32_t)(q + 1), k, est);
          if (cp[q])
            for (uint32_t kk = 1; kk <= cb.enc.Kmsbs + 1u; ++kk)
              tagtree_encode(pr.msbs, hdr, kk, k, est);
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
              pk.body_size += (uint32_t)(end - start);
            else
              pk.pieces.emplace_back(cb.data_off + start, (uint32_t)(end - start));
          }
        }
      }
    }
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

// create_quality_layer (tier2.c:896-1079), a packet at a time: the truncation points of the
// packet's codeblocks (every subband's precinct at that position), then the packet's header
static int64_t quality_layer_packet(const bwc_gl_ctrl &c, const PacketRef &r, uint16_t threshold,
                                    int q, uchar est) {
  Parameter &par = *r.par;
  Resolution &res = *r.res;
  const uint32_t p = r.p;
  int64_t size = 0;
  for (uint8_t m = 0; m < res.nsub; ++m) {
    const Subband &sb = par.subbands[res.first_subband + m];
    Precinct &pr = par.precincts[sb.first_precinct + p];
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
      if (cp[q] > cp[q - 1]) res.packets[(uint64_t)q * res.nprec + p].e = 1;
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
  }
  const int64_t ph = create_packet(par, res, p, q, est + 1);
  return (ph < 0) ? -1 : size + ph;
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

// byte count of a bit string written with BitWriter::emit and BitWriter::flush
struct StuffCounter {
  uint32_t T = 0;
  int t = 8;
  uint64_t bytes = 0;
  void put(uint64_t v, int n) {   // the n (<= 64) low bits of v, most significant first
    while (n > 0) {
      const int k = n < t ? n : t;
      const uint32_t chunk = (uint32_t)(v >> (n - k)) & ((1u << k) - 1u);
      T |= chunk << (t - k);
      t -= k;
      n -= k;
      if (t == 0) {
        bytes++;
        t = (T == 0xFF) ? 7 : 8;
        T = 0;
      }
    }
  }
  void put_bits(const RawBits &rb, uint64_t off, uint64_t n) {
    while (n) {
      const uint64_t b = off & 63;
      uint64_t m = 64 - b;
      if (m > n) m = n;
      if (m > 56) m = 56;
      const uint64_t v = (rb.words[off >> 6] << b) >> (64 - m);
      put(v, (int)m);
      off += m;
      n -= m;
    }
  }
  void put_ones(int n) {
    while (n > 0) {
      const int m = n < 32 ? n : 32;
      put((1ull << m) - 1, m);
      n -= m;
    }
  }
  uint64_t finish() const { return bytes + (t != 8 ? 1 : 0); }
};

struct ProbeCb {
  const Codeblock *cb;
  int16_t zprev;            // truncation point of the previous layer
  uint32_t rec_off, rec_n;  // slope records
  uint32_t pool;            // bit pool holding its tag-tree bits
  uint64_t incl_off, msbs_off;
  uint32_t incl_n, msbs_n;
};

struct ProbePacket {
  uint32_t first, count;
};

struct Probe {
  // right-to-left slope records of every codeblock: z in decreasing order with strictly
  // increasing S; max{z : S[z] >= t} is the first record whose S >= t
  std::vector<uint16_t> rec_s;
  std::vector<int16_t> rec_z;
  std::vector<uint32_t> rec_off;   // per codeblock in tile order (parameters concatenated)
  std::vector<ProbeCb> cbs;
  std::vector<ProbePacket> packets;
  std::vector<RawBits> pools;   // one per chunk of packets that built them
};

void build_records(Tile &tile, Probe &pr) {
  for (Parameter &par : tile.params)
    for (Codeblock &cb : par.codeblocks) {
      pr.rec_off.push_back((uint32_t)pr.rec_s.size());
      int best = -1;
      for (int z = cb.enc.Z; z >= 0; --z) {
        if ((int)cb.enc.S[z] > best) {
          best = cb.enc.S[z];
          pr.rec_s.push_back(cb.enc.S[z]);
          pr.rec_z.push_back((int16_t)z);
        }
      }
    }
  pr.rec_off.push_back((uint32_t)pr.rec_s.size());
}

// per-layer tables in the order create_packet visits codeblocks, built a chunk of packets at a
// time (each chunk has its own bit pool) and concatenated in packet order
void build_layer(Tile &tile, int q, Probe &pr) {
  const std::vector<PacketRef> pks = packet_list(tile);
  const size_t nchunks = std::min(pks.size(), WorkPool::instance().size() * 4);
  std::vector<std::vector<ProbeCb>> ccbs(nchunks);
  std::vector<std::vector<ProbePacket>> cpks(nchunks);
  pr.pools.assign(nchunks, RawBits());
  WorkPool::instance().run(nchunks, [&](size_t ch) {
    RawBits &pool = pr.pools[ch];
    for (size_t i = pks.size() * ch / nchunks; i < pks.size() * (ch + 1) / nchunks; ++i) {
      const PacketRef &r = pks[i];
      Parameter &par = *r.par;
      Resolution &res = *r.res;
      ProbePacket pk{(uint32_t)ccbs[ch].size(), 0};
      for (uint8_t m = 0; m < res.nsub; ++m) {
        const Subband &sb = par.subbands[res.first_subband + m];
        const Precinct &prc = par.precincts[sb.first_precinct + r.p];
        for (uint64_t k = 0; k < prc.ncb; ++k) {
          const uint64_t ci = prc.first_cb + k;
          Codeblock &cb = par.codeblocks[ci];
          ProbeCb e{};
          e.cb = &cb;
          e.zprev = cb.cp()[q - 1];
          e.rec_off = pr.rec_off[r.cb_base + ci];
          e.rec_n = pr.rec_off[r.cb_base + ci + 1] - e.rec_off;
          e.pool = (uint32_t)ch;
          if (e.zprev == 0) {
            e.incl_off = pool.n;
            tagtree_estimate(prc.incl, pool, (uint32_t)(q + 1), k);
            e.incl_n = (uint32_t)(pool.n - e.incl_off);
            e.msbs_off = pool.n;
            for (uint32_t kk = 1; kk <= cb.enc.Kmsbs + 1u; ++kk)
              tagtree_estimate(prc.msbs, pool, kk, k);
            e.msbs_n = (uint32_t)(pool.n - e.msbs_off);
          }
          ccbs[ch].push_back(e);
          pk.count++;
        }
      }
      cpks[ch].push_back(pk);
    }
  });
  pr.cbs.clear();
  pr.packets.clear();
  for (size_t ch = 0; ch < nchunks; ++ch) {
    const uint32_t base = (uint32_t)pr.cbs.size();
    for (ProbePacket pk : cpks[ch]) {
      pk.first += base;
      pr.packets.push_back(pk);
    }
    pr.cbs.insert(pr.cbs.end(), ccbs[ch].begin(), ccbs[ch].end());
  }
}

inline int16_t truncation_point(const Probe &pr, const ProbeCb &e, uint16_t threshold) {
  uint32_t lo = 0, hi = e.rec_n;   // first record with S >= threshold
  const uint16_t *s = pr.rec_s.data() + e.rec_off;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (s[mid] >= threshold) hi = mid; else lo = mid + 1;
  }
  return (lo < e.rec_n) ? pr.rec_z[e.rec_off + lo] : (int16_t)-1;
}

// create_quality_layer(codec, tile, threshold, q, 1) for the tables of layer q, over packets
// [first, last)
int64_t probe_packets(const Probe &pr, uint16_t threshold, size_t first, size_t last) {
  int64_t size = 0;
  for (size_t ip = first; ip < last; ++ip) {
    const ProbePacket &pk = pr.packets[ip];
    StuffCounter sc;
    sc.put(1, 1);
    bool e = false;
    for (uint32_t i = pk.first; i < pk.first + pk.count; ++i) {
      const ProbeCb &c = pr.cbs[i];
      const CodedBlock &enc = c.cb->enc;
      const int16_t z = truncation_point(pr, c, threshold);
      int16_t cpq;
      if (z < c.zprev) {
        cpq = c.zprev;
        if (cpq == 1) size += (int64_t)enc.L[0];
      } else {
        cpq = z;
        if (z > 0) {
          size += (int64_t)enc.L[z - 1];
          if (z > 1 && c.zprev > 0) size -= (int64_t)enc.L[c.zprev - 1];
        }
      }
      const int dz = cpq - c.zprev;
      if (dz > 0) e = true;
      if (c.zprev == 0) {
        sc.put_bits(pr.pools[c.pool], c.incl_off, c.incl_n);
        if (cpq) sc.put_bits(pr.pools[c.pool], c.msbs_off, c.msbs_n);
      } else {
        sc.put(dz ? 1 : 0, 1);
      }
      if (!dz) continue;
      // encode_delta_z
      if (dz == 1) sc.put(0, 1);
      else if (dz == 2) sc.put(2, 2);
      else if (dz < 6) sc.put(12u | (uint32_t)(dz - 3), 4);
      else if (dz < 37) sc.put((15u << 5) | (uint32_t)(dz - 6), 9);
      else if (dz < 293) sc.put((511u << 8) | (uint32_t)(dz - 37), 17);
      // encode_length with the estimate state
      const int16_t z_curr = cpq - 1, z_prev = c.zprev - 1;
      const uint16_t beta = c.cb->beta_est;
      uint16_t max_beta = beta;
      const uint32_t L = (uint32_t)(enc.L[z_curr] - ((z_prev >= 0) ? enc.L[z_prev] : 0));
      const uint16_t cp_bits = ilog2_u16((uint64_t)(z_curr - z_prev));
      const int32_t L_bits = (int32_t)ilog2_u16(L) + 1 - cp_bits;
      max_beta = (max_beta < L_bits) ? (uint16_t)L_bits : max_beta;
      sc.put_ones(max_beta - beta);
      sc.put(0, 1);
      const int sh = max_beta + cp_bits - 1;
      if (sh >= 0 && sh < 31) sc.put(L & (uint32_t)((2ull << sh) - 1), sh + 1);
    }
    size += e ? (int64_t)sc.finish() : 1;
  }
  return size;
}

// probe_packets for several thresholds at once: every (threshold, chunk of packets) pair is a
// task on the pool
void probe_thresholds(const Probe &pr, const std::vector<uint16_t> &thr, std::vector<int64_t> &out) {
  const size_t np = pr.packets.size(), nt = thr.size();
  const size_t chunks = std::max<size_t>(1, std::min(np, WorkPool::instance().size() * 4 / nt + 1));
  std::vector<int64_t> part(nt * chunks, 0);
  WorkPool::instance().run(nt * chunks, [&](size_t i) {
    const size_t k = i / chunks, c = i % chunks;
    part[i] = probe_packets(pr, thr[k], np * c / chunks, np * (c + 1) / chunks);
  });
  out.assign(nt, 0);
  for (size_t i = 0; i < nt * chunks; ++i) out[i / chunks] += part[i];
}

}  // namespace

// ---- rate-control warm start ---------------------------------------------------------------
// The reference's per-layer bisection (tier2.c:1115-1254) is a chain of dependent probes, each
// a full truncation-and-header estimate.  Its outcome depends on the exact sequence of probes,
// so the search itself is kept: the same probes, compared the same way, in the same order.
// What a predicted final threshold changes is WHEN the probes are evaluated: from the
// prediction the whole probe path is simulated (assuming the size falls as the threshold
// rises) and evaluated at once, in parallel host threads; the exact bisection then replays over
// those results, and only when its path leaves the predicted one is a new round needed (again
// speculated from the prediction).  The selected slope, and so every output byte, is the
// plain search's; what the prediction saves is rounds of dependent probes.
//
// Features of one layer (kRateFeatures values): a 32-bin histogram (fractions) of the
// codeblocks' non-zero pass slopes S[1..Z] over the 16-bit log range, log(bits per value of the
// layer) / 4 and (log(values) - 14) / 4.  The network predicts the final slope / 65536.

namespace {

void rate_features(const Tile &tile, float bpv, float *out) {
  double hist[32] = {};
  double total = 0;
  for (const Parameter &par : tile.params)
    for (const Codeblock &cb : par.codeblocks)
      for (int z = 1; z <= cb.enc.Z; ++z)
        if (cb.enc.S[z]) {
          hist[cb.enc.S[z] >> 11] += 1;
          total += 1;
        }
  for (int i = 0; i < 32; ++i) out[i] = total > 0 ? (float)(hist[i] / total) : 0.f;
  uint64_t values = tile.box.size() * tile.params.size();
  out[32] = (float)(std::log((double)std::max(bpv, 1e-6f)) / 4.0);
  out[33] = (float)((std::log((double)std::max<uint64_t>(values, 1)) - 14.0) / 4.0);
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
  for (uint8_t l = 0; l < c.nLayers; ++l)
    rate_features(tile, c.bitrate[l], tile.rc_features.data() + (size_t)l * kRateFeatures);
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
    est = create_quality_layer(codec, tile, slope, l, 0);
    if (est >= 0)
      est_tile += est + (int64_t)header_size;
    else
      return 1;
  }
  return 0;
}

// create_packets (tier2.c:751-849): final headers for every packet, then the per-codeblock
// coding state is cleared as in the reference.
static uchar create_packets(bwc_codec *codec, Tile &tile) {
  const bwc_gl_ctrl &c = codec->control;
  const std::vector<PacketRef> pks = packet_list(tile);
  std::atomic<bool> bad{false};
  for_chunks(pks.size(), [&](size_t first, size_t last) {
    for (size_t i = first; i < last; ++i) {
      Parameter &par = *pks[i].par;
      Resolution &res = *pks[i].res;
      const uint32_t p = pks[i].p;
      for (uint8_t l = 0; l < c.nLayers; ++l)
        if (create_packet(par, res, p, l, 0) < 0) bad = true;
      // the reference clears each codeblock's coding state once its packets exist
      for (uint8_t m = 0; m < res.nsub; ++m) {
        const Subband &sb = par.subbands[res.first_subband + m];
        const Precinct &pr = par.precincts[sb.first_precinct + p];
        for (uint64_t k = 0; k < pr.ncb; ++k) {
          Codeblock &cb = par.codeblocks[pr.first_cb + k];
          cb.enc = CodedBlock();
          for (int l = 0; l < c.nLayers; ++l) cb.cp()[l] = 0;
        }
      }
    }
  });
  return bad ? 1 : 0;
}

uchar t2_encode(bwc_codec *codec, Tile &tile) {
  if (create_quality_layers(codec, tile)) return 1;
  if (create_packets(codec, tile)) return 1;
  return 0;
}

static void decode_length(BitReader &br, Codeblock &cb, int q) {
  while (br.get_bit()) cb.beta++;
  int16_t *cp = cb.cp();
  const int16_t z_curr = cp[q] - 1, z_prev = cp[q - 1] - 1;
  uint16_t L_bits = (uint16_t)(cb.beta + ilog2_u16((uint64_t)(z_curr - z_prev)));
  uint32_t i = 0;
  for (; L_bits > 0; --L_bits) {
    i <<= 1;
    i |= br.get_bit();
  }
  cb.enc.L[z_curr] = ((z_prev >= 0) ? cb.enc.L[z_prev] : 0) + i;
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
            uint32_t kk = 1;
            while (tagtree_decode(pr.msbs, br, kk++, k)) {
            }
            cb.enc.Kmsbs = (uint8_t)pr.msbs.nodes[k].value;
          }
        } else {
          dz = br.get_bit();
        }
        cp[q] = cp[q - 1];
        if (dz) {
          dz = decode_delta_z(br);
          cp[q] += dz;
          cb.enc.Z = (uint8_t)cp[q];
          decode_length(br, cb, q);
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
