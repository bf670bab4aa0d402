// bwc_compress / bwc_decompress: the device pipeline behind the libbwc API.
//
// Compression of one tile (libbwc.c:3145-3438), per parameter, all on the codec's CUDA stream:
//   upload -> fill + min/max -> normalise -> forward 9/7 DWT -> tier-1 encode (warp per
//   codeblock); then one download of the per-codeblock tier-1 summary (K, Z, truncation
//   lengths, log slopes), host tier-2 (rate control, packet headers, layout), and one device
//   gather that assembles header bytes and coded-byte slices into the codestream, which is
//   copied to stream->out.
// Decompression (libbwc.c:3485-3710): host parsing of headers and packets, upload of the
// codestream, device gather of each codeblock's bytes, tier-1 decode + dequantise, inverse DWT,
// denormalise + dtype conversion, copy to stream->out.
//
// There is no CPU fallback: a missing or failing GPU makes the calls fail (0 / 1 returns and a
// diagnostic on stderr, the reference's error convention).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../kernels/kernels.hpp"
#include "bwc_b200.h"
#include "common.hpp"

namespace bwcb {

namespace {

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  fprintf(stderr,
          "o##########################################################o\n"
          "| ERROR: CUDA failure in %-34s|\n"
          "|        %-50s|\n"
          "o##########################################################o\n",
          what, cudaGetErrorString(e));
  return false;
}

// Process-wide cache of device allocations: codecs are short-lived (one per field in the
// libbwc usage pattern), so their buffers are recycled instead of cudaMalloc'd per call.
class Pool {
 public:
  static Pool &get() {
    static Pool p;
    return p;
  }
  void *acquire(size_t bytes, size_t *got) {
    std::lock_guard<std::mutex> l(m_);
    auto it = free_.lower_bound(bytes);
    if (it != free_.end() && it->first <= bytes * 2 + (1 << 20)) {
      void *p = it->second;
      *got = it->first;
      free_.erase(it);
      return p;
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      // give cached blocks back and retry once
      for (auto &kv : free_) cudaFree(kv.second);
      free_.clear();
      cudaGetLastError();
      if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
    }
    *got = bytes;
    return p;
  }
  void release(void *p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> l(m_);
    free_.emplace(bytes, p);
  }

 private:
  std::mutex m_;
  std::multimap<size_t, void *> free_;
};

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  template <typename T>
  T *as() const { return reinterpret_cast<T *>(p); }
  bool ensure(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (cap >= bytes) return true;
    Pool::get().release(p, cap);
    p = Pool::get().acquire(bytes, &cap);
    if (!p) {
      cap = 0;
      fprintf(stderr, "%s", kMemError);
      return false;
    }
    return true;
  }
  void drop() {
    Pool::get().release(p, cap);
    p = nullptr;
    cap = 0;
  }
};

// Page-locked host memory, grown as needed and kept (copies from the device into it run at
// full DMA speed; the driver stages copies into pageable memory through small chunks).
struct PinnedBuf {
  void *p = nullptr;
  size_t cap = 0;
  bool ensure(size_t bytes) {
    if (cap >= bytes) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return false;
    }
    cap = bytes;
    return true;
  }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

// Page-locked tier-1 result buffer of each device, shared by the process's codecs (a codec's
// own would be allocated, slowly, by every new codec); held under its mutex while a call copies
// its results in and reads them out.  Kept until the process ends.
std::mutex g_t1host_mutex[64];
PinnedBuf *g_t1host[64] = {};

PinnedBuf &t1host_of(int dev) {
  if (!g_t1host[dev]) g_t1host[dev] = new PinnedBuf();   // under g_t1host_mutex[dev]
  return *g_t1host[dev];
}

// Host copy of the tier-1 results of one call: per codeblock K, Z, truncation lengths, slopes
// and flags, per slope slot the slope range, per unit the field statistics.  Lives in the
// caller's page-locked buffer, or in `fallback` when no page-locked memory can be had.
struct T1Host {
  uint8_t *K = nullptr, *Z = nullptr;
  uint32_t *L = nullptr, *flags = nullptr, *slopes = nullptr;
  uint16_t *S = nullptr;
  bwc_float *stats = nullptr;
  uint32_t *fault = nullptr;   // the transform's fault word
  std::vector<uint8_t> fallback;
  bool layout(PinnedBuf &pb, uint64_t ncb, uint64_t nslots, uint64_t nu) {
    auto al = [](uint64_t x) { return (x + 15) & ~15ull; };
    const uint64_t oZ = al(ncb), oL = oZ + al(ncb), oF = oL + al(ncb * kMaxPasses * 4),
                   oSl = oF + al(ncb * 4), oS = oSl + al(8 * nslots),
                   oSt = oS + al(ncb * (kMaxPasses + 1) * 2),
                   oFa = oSt + al(4 * sizeof(bwc_float) * nu), end = oFa + 16;
    uint8_t *base = nullptr;
    if (pb.ensure(end)) {
      base = static_cast<uint8_t *>(pb.p);
    } else {
      fallback.assign(end + 16, 0);
      base = reinterpret_cast<uint8_t *>(
          (reinterpret_cast<uintptr_t>(fallback.data()) + 15) & ~uintptr_t(15));
    }
    K = base;
    Z = base + oZ;
    L = reinterpret_cast<uint32_t *>(base + oL);
    flags = reinterpret_cast<uint32_t *>(base + oF);
    slopes = reinterpret_cast<uint32_t *>(base + oSl);
    S = reinterpret_cast<uint16_t *>(base + oS);
    stats = reinterpret_cast<bwc_float *>(base + oSt);
    fault = reinterpret_cast<uint32_t *>(base + oFa);
    return true;
  }
};

uint8_t sig_class(uint8_t hb) {
  // context table by subband orientation (tier1.c:2416-2446)
  switch (hb) {
    case 1: case 5: case 9: case 13: return 1;
    case 3: case 7: case 11: case 15: return 2;
    default: return 0;
  }
}

}  // namespace

struct DeviceState {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  DevBuf temp;     // second field-sized buffer: the transform reads one and writes the other
  DevBuf in, work, keys, stats, cbtab, sbtab, bytes, scratch, snaps, dmse, K, Z, L, S, flags,
      slopes, counter, cs, blob, pieces, outbuf, mags, lmax, symbols, pcount, poff, symused,
      order, queue;
  bool dump_set = false, ddump_set = false;
  bwc_b200_stage_dump dump{};
  bwc_b200_decode_dump ddump{};
  double timings[12] = {};   // stage times (ms); [8] tier-1 symbols coded (millions),
                             // [9] tier-1 context modelling (ms, part of [3]), [10] the MQ
                             // launches' device time summed (ms), [11] MQ launches

  ~DeviceState() {
    DevBuf *all[] = {&order, &queue, &temp, &in, &work, &keys, &stats, &cbtab, &sbtab, &bytes, &scratch, &snaps, &dmse,
                     &K, &Z, &L, &S, &flags, &slopes, &counter, &cs, &blob, &pieces, &outbuf,
                     &mags, &lmax, &symbols, &pcount, &poff, &symused};
    if (stream) cudaStreamSynchronize(stream);
    for (DevBuf *b : all) b->drop();
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
};

static DeviceState *device_state(bwc_codec *codec) {
  bwc_b200_engine *eng = codec->tile;
  if (!eng) return nullptr;
  if (!eng->dev) {
    DeviceState *d = new (std::nothrow) DeviceState();
    if (!d) return nullptr;
    if (!cuda_ok(cudaGetDevice(&d->device), "cudaGetDevice") ||
        !cuda_ok(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "stream")) {
      delete d;
      return nullptr;
    }
    for (auto &e : d->ev) cudaEventCreate(&e);
    eng->dev = d;
  }
  return eng->dev;
}

void free_engine(bwc_codec *codec) {
  if (!codec || !codec->tile) return;
  delete codec->tile->dev;
  delete codec->tile;
  codec->tile = nullptr;
}

// timing events of one stage sequence, released however the scope is left
// MQ launch timing events of one tier-1 launch
struct ScopedMqTimes {
  T1LaunchTimes t;
  ScopedMqTimes() {
    for (int i = 0; i < 8; ++i) {
      cudaEventCreate(&t.start[i]);
      cudaEventCreate(&t.end[i]);
    }
  }
  ~ScopedMqTimes() {
    for (int i = 0; i < 8; ++i) {
      cudaEventDestroy(t.start[i]);
      cudaEventDestroy(t.end[i]);
    }
  }
  double total_ms() const {
    double sum = 0;
    for (int i = 0; i < t.n; ++i) {
      float x = 0;
      if (cudaEventElapsedTime(&x, t.start[i], t.end[i]) == cudaSuccess) sum += x;
    }
    cudaGetLastError();
    return sum;
  }
  ScopedMqTimes(const ScopedMqTimes &) = delete;
  ScopedMqTimes &operator=(const ScopedMqTimes &) = delete;
};

struct ScopedEvents {
  cudaEvent_t e[5];
  ScopedEvents() {
    for (auto &x : e) cudaEventCreate(&x);
  }
  ~ScopedEvents() {
    for (auto &x : e) cudaEventDestroy(x);
  }
  ScopedEvents(const ScopedEvents &) = delete;
  ScopedEvents &operator=(const ScopedEvents &) = delete;
};

// host memory that is page-locked (registered with or allocated by CUDA)
static bool is_pinned_host(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static bool is_device_pointer(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Copies between pageable host memory and the device through two page-locked chunks kept per
// device: host threads fill (or empty) one chunk while the copy engine moves the other.  A copy
// straight from or to pageable memory is staged by the driver through small buffers of its
// own, several times slower.  Page-locked host memory is copied directly, and so is everything
// when the chunks are in use by another call or cannot be allocated.
class HostStaging {
 public:
  static constexpr uint64_t kChunk = 32ull << 20;
  static constexpr uint64_t kMinBytes = 4ull << 20;   // smaller copies go directly

  static HostStaging *for_device(int device) {
    static std::mutex m;
    static std::map<int, HostStaging *> all;   // kept for the process's lifetime
    std::lock_guard<std::mutex> l(m);
    HostStaging *&h = all[device];
    if (!h) h = new (std::nothrow) HostStaging();
    return h;
  }

  // host -> device; returns false (nothing copied) when the caller should copy directly
  bool upload(void *dst, const void *src, uint64_t n, cudaStream_t s) {
    std::unique_lock<std::mutex> busy(m_, std::try_to_lock);
    if (!busy.owns_lock() || n < kMinBytes || is_pinned_host(src) || !ready()) return false;
    for (uint64_t off = 0, k = 0; off < n; off += kChunk, ++k) {
      const int h = (int)(k & 1);
      const uint64_t len = std::min(kChunk, n - off);
      cudaEventSynchronize(done_[h]);   // the copy that last read this chunk has finished
      fill(buf_[h], static_cast<const uint8_t *>(src) + off, len);
      if (cudaMemcpyAsync(static_cast<uint8_t *>(dst) + off, buf_[h], len,
                          cudaMemcpyHostToDevice, s) != cudaSuccess)
        return fail();
      cudaEventRecord(done_[h], s);
    }
    return true;
  }

  // device -> host, complete on return; false (nothing copied) when the caller should copy
  // directly
  bool download(void *dst, const void *src, uint64_t n, cudaStream_t s) {
    std::unique_lock<std::mutex> busy(m_, std::try_to_lock);
    if (!busy.owns_lock() || n < kMinBytes || is_pinned_host(dst) || !ready()) return false;
    uint64_t prev_off = 0, prev_len = 0;
    for (uint64_t off = 0, k = 0;; off += kChunk, ++k) {
      const int h = (int)(k & 1);
      const uint64_t len = off < n ? std::min(kChunk, n - off) : 0;
      if (len) {
        cudaEventSynchronize(done_[h]);
        if (cudaMemcpyAsync(buf_[h], static_cast<const uint8_t *>(src) + off, len,
                            cudaMemcpyDeviceToHost, s) != cudaSuccess)
          return fail();
        cudaEventRecord(done_[h], s);
      }
      if (prev_len) {   // while chunk k moves, empty chunk k - 1
        if (cudaEventSynchronize(done_[h ^ 1]) != cudaSuccess) return fail();
        fill(static_cast<uint8_t *>(dst) + prev_off, buf_[h ^ 1], prev_len);
      }
      if (!len) break;
      prev_off = off;
      prev_len = len;
    }
    return true;
  }

 private:
  bool ready() {
    if (buf_[0]) return true;
    if (failed_) return false;
    for (int h = 0; h < 2; ++h)
      if (cudaHostAlloc(&buf_[h], kChunk, cudaHostAllocPortable) != cudaSuccess ||
          cudaEventCreateWithFlags(&done_[h], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        for (int j = 0; j < 2; ++j) {
          if (buf_[j]) cudaFreeHost(buf_[j]);
          if (done_[j]) cudaEventDestroy(done_[j]);
          buf_[j] = nullptr;
          done_[j] = nullptr;
        }
        failed_ = true;
        return false;
      }
    return true;
  }
  static bool fail() {   // a copy could not be queued: the caller copies directly (and reports)
    cudaGetLastError();
    return false;
  }
  // one chunk, in slices on the host thread pool
  static void fill(void *dst, const void *src, uint64_t len) {
    constexpr uint64_t kSlice = 2ull << 20;
    const size_t ns = (size_t)((len + kSlice - 1) / kSlice);
    host_parallel(ns, [&](size_t i) {
      const uint64_t a = i * kSlice, b = std::min(len, a + kSlice);
      std::memcpy(static_cast<uint8_t *>(dst) + a, static_cast<const uint8_t *>(src) + a, b - a);
    });
  }
  std::mutex m_;
  void *buf_[2] = {nullptr, nullptr};
  cudaEvent_t done_[2] = {nullptr, nullptr};
  bool failed_ = false;
};

static DwtPlan make_plan(const bwc_gl_ctrl &c, const Parameter &par) {
  DwtPlan plan{};
  plan.levels = c.nDecomp;
  const uint8_t dec[4] = {c.decompX, c.decompY, c.decompZ, c.decompTS};
  const uint8_t kern[4] = {(uint8_t)c.KernelX, (uint8_t)c.KernelY, (uint8_t)c.KernelZ,
                           (uint8_t)c.KernelTS};
  for (int a = 0; a < 4; ++a) plan.kern[a] = (kern[a] == bwc_dwt_5_3) ? 1 : 0;
  for (int l = 0; l < c.nDecomp; ++l) {
    const Box &b = par.res[c.nDecomp - l].box;
    const uint64_t e[4] = {b.X1 - b.X0, b.Y1 - b.Y0, b.Z1 - b.Z0, b.TS1 - b.TS0};
    const uint64_t o[4] = {b.X0, b.Y0, b.Z0, b.TS0};
    for (int a = 0; a < 4; ++a) {
      plan.ext[l][a] = e[a];
      if (l < dec[a] && e[a] > 1) plan.axis_on[l] |= (uint8_t)(1 << a);
      if (o[a] & 1) plan.odd[l] |= (uint8_t)(1 << a);
    }
  }
  return plan;
}

// Codeblock and subband tables of one parameter whose working buffer has the extents `dims`
// (codeblocks address it from element 0, slope range slot 0).
static void build_tables(const Parameter &par, const FieldDims &dims, uchar erres, bool compress,
                         std::vector<CbDev> &cbs, std::vector<SbDev> &sbs, uint64_t *bytes_total,
                         uint64_t *scratch_total, uint32_t *max_cols) {
  sbs.clear();
  for (const Subband &s : par.subbands) {
    SbDev d;
    double g = (double)s.dwt_gain;
    g *= (double)(bwc_float)(s.qt_step * s.qt_step);
    d.gain_step2 = g;
    d.qt_eff = s.qt_eff;
    d.Kmax = s.Kmax;
    d.cls = sig_class(s.highband);
    d.erres = erres ? 1u : 0u;
    d.pad = 0;
    sbs.push_back(d);
  }
  cbs.clear();
  uint64_t off = 0, soff = 0;
  uint32_t mc = 0;
  for (const Codeblock &cb : par.codeblocks) {
    CbDev d;
    d.x0 = (uint32_t)cb.box.X0;
    d.y0 = (uint32_t)cb.box.Y0;
    d.z0 = (uint32_t)cb.box.Z0;
    d.t0 = (uint32_t)cb.box.TS0;
    d.w = (uint32_t)(cb.box.X1 - cb.box.X0);
    d.h = (uint32_t)(cb.box.Y1 - cb.box.Y0);
    d.d = (uint32_t)(cb.box.Z1 - cb.box.Z0);
    d.nt = (uint32_t)(cb.box.TS1 - cb.box.TS0);
    d.sb = cb.subband;
    d.base = 0;
    d.sy = dims.width;
    d.sz = dims.width * dims.height;
    d.st = dims.width * dims.height * dims.depth;
    d.slot = 0;
    d.pad = 0;
    const uint64_t nsamp = (uint64_t)d.w * d.h * d.d * d.nt;
    const uint32_t ncols = d.w * ((d.h + 3) / 4) * d.d * d.nt;
    mc = std::max(mc, ncols);
    if (compress) {
      const uint64_t cap = nsamp * (kPrecByte + 1) + 64;
      d.out_off = off;
      d.out_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFF0u);
      off += (cap + 15) & ~15ull;
      d.scratch_off = soff;
      soff += t1_scratch_bytes(ncols);
    } else {
      d.out_off = 0;   // filled by the caller
      d.out_cap = 0;
      d.scratch_off = soff;   // elements of the decode scratch
      soff += t1_decode_scratch_elems(ncols);
    }
    cbs.push_back(d);
  }
  *bytes_total = off;
  *scratch_total = soff;
  *max_cols = mc;
}

// Codeblock indices [0, count) of cbs[first ...] sorted by expected tier-1 work (stripe columns x
// the subband's Kmax), largest first; ties keep tier-1 order.
static std::vector<uint32_t> work_order(const std::vector<CbDev> &cbs, const std::vector<SbDev> &sbs,
                                        size_t first, size_t count) {
  std::vector<uint32_t> order(count);
  std::vector<uint64_t> cost(count);
  for (size_t i = 0; i < count; ++i) {
    const CbDev &d = cbs[first + i];
    order[i] = (uint32_t)i;
    cost[i] = (uint64_t)d.w * ((d.h + 3) / 4) * d.d * d.nt * (sbs[d.sb].Kmax + 1);
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  return order;
}

static int t1_grid(const void *kernel_unused, size_t smem_per_block) {
  (void)kernel_unused;
  int dev = 0, sms = 148, smem_max = 227 * 1024;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  int per_sm = (int)std::max<size_t>(1, std::min<size_t>(16, smem_max / (smem_per_block + 1024)));
  return sms * per_sm;
}

// ---------------------------------------------------------------------------------------------
// One tile of one parameter: the unit the device pipeline runs through (a single-tile field has
// one unit per parameter).  Tiles are taken in tile order, within a tile parameter by parameter,
// as the reference codes them (libbwc.c:3231-3358).
struct TileUnit {
  uint32_t tile, param;
  FieldDims dims;      // the tile's extent
  uint64_t n;          // samples of the tile
  BoxMap map;          // where the tile's samples sit in the user's field
  bool whole;          // the tile is the whole field (contiguous)
};

// The tiles of a codec as units.  A tile's samples are read from (and written back to) the
// field at X0 + nX * (Y0 + y + nY * (Z0 + z + nZ * t)) + the parameter's offset, with t counted
// from the field's first time step, not the tile's (the reference's fill_buffer and
// flush_buffer, libbwc.c:727-729 and :870-875, index with t, not TS0 + t).
static std::vector<TileUnit> tile_units(const bwc_codec *codec) {
  const bwc_gl_inf &info = codec->info;
  std::vector<TileUnit> units;
  const std::vector<Tile> &tiles = codec->tile->tiles;
  const bool single = tiles.size() == 1;
  for (const Tile &tile : tiles) {
    for (uint32_t p = 0; p < (uint32_t)info.nPar; ++p) {
      TileUnit u;
      u.tile = tile.index;
      u.param = p;
      u.dims = FieldDims{tile.box.nx(), tile.box.ny(), tile.box.nz(), tile.box.nt()};
      u.n = tile.box.size();
      const uint64_t po = info.nX * info.nY * info.nZ * info.nTS * (uint64_t)p;
      u.map.w = u.dims.width;
      u.map.h = u.dims.height;
      u.map.d = u.dims.depth;
      u.map.sy = info.nX;
      u.map.sz = info.nX * info.nY;
      u.map.st = info.nX * info.nY * info.nZ;
      u.map.base = po + tile.box.X0 + info.nX * (tile.box.Y0 + info.nY * tile.box.Z0);
      u.whole = single;
      units.push_back(u);
    }
  }
  return units;
}

static size_t compress_impl(bwc_codec *codec, bwc_stream *stream) {
  bwc_b200_engine *eng = codec->tile;
  if (!eng || eng->tiles.empty()) {
    warn("o##########################################################o\n"
         "| ERROR: bwc_create_compression has not been called        |\n"
         "o##########################################################o\n");
    return 0;
  }
  DeviceState *dv = device_state(codec);
  if (!dv) return 0;
  cudaStream_t s = dv->stream;
  bwc_gl_ctrl &c = codec->control;
  bwc_gl_inf &info = codec->info;
  const size_t dsz = (info.data_prec == bwc_precision_double) ? 8 : 4;
  const uint64_t in_bytes = info.nX * info.nY * info.nZ * info.nTS * (uint64_t)info.nPar * dsz;
  const std::vector<TileUnit> units = tile_units(codec);
  const size_t nu = units.size();
  const size_t ntiles = eng->tiles.size();
  uint64_t nmax = 0;
  for (const TileUnit &u : units) nmax = std::max(nmax, u.n);

  cudaEventRecord(dv->ev[0], s);
  const uint8_t *src = (const uint8_t *)stream->inp;
  if (!is_device_pointer(stream->inp)) {
    if (!dv->in.ensure(in_bytes)) return 0;
    HostStaging *hs = HostStaging::for_device(dv->device);
    if (!(hs && hs->upload(dv->in.p, stream->inp, in_bytes, s)) &&
        !cuda_ok(cudaMemcpyAsync(dv->in.p, stream->inp, in_bytes, cudaMemcpyHostToDevice, s), "upload"))
      return 0;
    src = dv->in.as<uint8_t>();
  }
  cudaEventRecord(dv->ev[1], s);

  // tables and output regions of every unit; a codeblock's slope range goes to its tile's slot
  std::vector<std::vector<CbDev>> cbs(nu);
  std::vector<std::vector<SbDev>> sbs(nu);
  std::vector<uint64_t> cb_base(nu + 1, 0), byte_base(nu + 1, 0), scr_base(nu + 1, 0),
      sb_base(nu + 1, 0);
  uint32_t max_cols = 0;
  for (size_t ui = 0; ui < nu; ++ui) {
    const TileUnit &u = units[ui];
    uint64_t bt, st;
    uint32_t mc;
    build_tables(eng->tiles[u.tile].params[u.param], u.dims, c.error_resilience, true, cbs[ui],
                 sbs[ui], &bt, &st, &mc);
    max_cols = std::max(max_cols, mc);
    cb_base[ui + 1] = cb_base[ui] + cbs[ui].size();
    byte_base[ui + 1] = byte_base[ui] + bt;
    scr_base[ui + 1] = scr_base[ui] + st;
    sb_base[ui + 1] = sb_base[ui] + sbs[ui].size();
    for (CbDev &d : cbs[ui]) {
      d.out_off += byte_base[ui];
      d.scratch_off += scr_base[ui];
      d.sb += (uint32_t)sb_base[ui];
      d.slot = u.tile;
    }
  }
  const uint64_t ncb = cb_base[nu];
  std::vector<CbDev> allcb;
  std::vector<SbDev> allsb;
  for (size_t ui = 0; ui < nu; ++ui) {
    allcb.insert(allcb.end(), cbs[ui].begin(), cbs[ui].end());
    allsb.insert(allsb.end(), sbs[ui].begin(), sbs[ui].end());
  }
  if (!dv->work.ensure(nmax * sizeof(bwc_float)) || !dv->temp.ensure(nmax * sizeof(bwc_float)) ||
      !dv->keys.ensure(16 * nu) || !dv->stats.ensure(4 * sizeof(bwc_float) * nu) ||
      !dv->cbtab.ensure(sizeof(CbDev) * ncb) || !dv->sbtab.ensure(sizeof(SbDev) * allsb.size()) ||
      !dv->bytes.ensure(byte_base[nu]) || !dv->scratch.ensure(scr_base[nu]) ||
      !dv->snaps.ensure(ncb * kMaxPasses * 16) || !dv->dmse.ensure(ncb * kMaxPasses * 8) ||
      !dv->K.ensure(ncb) || !dv->Z.ensure(ncb) || !dv->L.ensure(ncb * kMaxPasses * 4) ||
      !dv->S.ensure(ncb * (kMaxPasses + 1) * 2) || !dv->flags.ensure(ncb * 4) ||
      !dv->slopes.ensure(8 * ntiles) || !dv->counter.ensure(4 * nu))
    return 0;
  cudaMemcpyAsync(dv->cbtab.p, allcb.data(), sizeof(CbDev) * ncb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dv->sbtab.p, allsb.data(), sizeof(SbDev) * allsb.size(), cudaMemcpyHostToDevice, s);
  {
    std::vector<uint32_t> init(2 * ntiles);
    for (size_t t = 0; t < ntiles; ++t) {
      init[2 * t] = 0xFFFF;
      init[2 * t + 1] = 0;
    }
    cudaMemcpyAsync(dv->slopes.p, init.data(), 8 * ntiles, cudaMemcpyHostToDevice, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "tier-1 tables")) return 0;   // `init` dies here
  }
  cudaMemsetAsync(dv->flags.p, 0, ncb * 4, s);
  cudaMemsetAsync(dv->counter.p, 0, 4 * nu, s);
  cudaMemsetAsync(dv->keys.p, 0, 16 * nu, s);
  for (size_t ui = 0; ui < nu; ++ui) cudaMemsetAsync(dv->keys.as<uint64_t>() + 2 * ui, 0xFF, 8, s);

  if (t1_model_smem(max_cols) > 200 * 1024) {
    warn("o##########################################################o\n"
         "| ERROR: codeblocks above 2^18 samples are not supported   |\n"
         "o##########################################################o\n");
    return 0;
  }
  // symbol arena: sized for about 1.1 symbols per sample and bit plane; a full arena is
  // detected per codeblock and the unit is coded again with a larger one
  uint64_t total_samples = 0;
  for (uint64_t i = 0; i < ncb; ++i)
    total_samples += (uint64_t)allcb[i].w * ((allcb[i].h + 3) / 4) * 4 * allcb[i].d * allcb[i].nt;
  uint64_t arena = std::max<uint64_t>(1 << 20, total_samples * (kPrecBit + 1) * 9 / 8);
  if (!dv->pcount.ensure(ncb * kMaxPasses * 4) || !dv->poff.ensure(ncb * kMaxPasses * 8) ||
      !dv->symused.ensure(16) || !dv->order.ensure(ncb * 4) || !dv->queue.ensure(32))
    return 0;
  {
    std::vector<uint32_t> order;
    for (size_t ui = 0; ui < nu; ++ui) {
      const std::vector<uint32_t> o = work_order(allcb, allsb, cb_base[ui], cbs[ui].size());
      order.insert(order.end(), o.begin(), o.end());
    }
    cudaMemcpyAsync(dv->order.p, order.data(), ncb * 4, cudaMemcpyHostToDevice, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "tier-1 order")) return 0;
  }
  float t_norm = 0, t_dwt = 0, t_t1 = 0, t_model = 0;
  double t_mq = 0;
  int mq_launches = 0;
  dv->timings[8] = 0;
  for (size_t ui = 0; ui < nu; ++ui) {
    const TileUnit &u = units[ui];
    Tile &tile = eng->tiles[u.tile];
    const ScopedEvents evs;
    cudaEvent_t a = evs.e[0], b2 = evs.e[1], c2 = evs.e[2], d2 = evs.e[3], m2 = evs.e[4];
    cudaEventRecord(a, s);
    if (u.whole)
      launch_fill_minmax(src + (uint64_t)u.param * u.n * dsz, dsz == 8, u.n,
                         dv->temp.as<bwc_float>(), dv->keys.as<uint64_t>() + 2 * ui, s);
    else
      launch_fill_minmax_box(src, dsz == 8, u.n, u.map, dv->temp.as<bwc_float>(),
                             dv->keys.as<uint64_t>() + 2 * ui, s);
    launch_normalize(dv->temp.as<bwc_float>(), u.n, dv->keys.as<uint64_t>() + 2 * ui, c.Qm,
                     dv->stats.as<bwc_float>() + 4 * ui, s);
    if (ui == 0 && dv->dump_set && dv->dump.normalized)
      cudaMemcpyAsync(dv->dump.normalized, dv->temp.p, u.n * sizeof(bwc_float), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(b2, s);
    launch_dwt_forward(dv->work.as<bwc_float>(), dv->temp.as<bwc_float>(), u.dims,
                       make_plan(c, tile.params[u.param]), s);
    if (ui == 0 && dv->dump_set && dv->dump.transformed)
      cudaMemcpyAsync(dv->dump.transformed, dv->work.p, u.n * sizeof(bwc_float), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(c2, s);
    T1EncOut o;
    o.bytes = dv->bytes.as<uint8_t>();
    o.K = dv->K.as<uint8_t>() + cb_base[ui];
    o.Z = dv->Z.as<uint8_t>() + cb_base[ui];
    o.L = dv->L.as<uint32_t>() + cb_base[ui] * kMaxPasses;
    o.S = dv->S.as<uint16_t>() + cb_base[ui] * (kMaxPasses + 1);
    o.slopes = dv->slopes.as<uint32_t>();
    o.flags = dv->flags.as<uint32_t>() + cb_base[ui];
    o.planes = dv->scratch.as<uint8_t>();
    o.snaps = dv->snaps.as<uint64_t>() + cb_base[ui] * kMaxPasses * 2;
    o.dmse = dv->dmse.as<int64_t>() + cb_base[ui] * kMaxPasses;
    o.pass_count = dv->pcount.as<uint32_t>() + cb_base[ui] * kMaxPasses;
    o.pass_off = dv->poff.as<uint64_t>() + cb_base[ui] * kMaxPasses;
    o.sym_used = dv->symused.as<unsigned long long>();
    ScopedMqTimes mqt;
    for (int attempt = 0;; ++attempt) {
      if (!dv->symbols.ensure(arena + 256)) return 0;
      o.symbols = dv->symbols.as<uint8_t>();
      o.sym_cap = dv->symbols.cap - 256;   // slack for the MQ kernel's read-ahead
      cudaMemsetAsync(dv->symused.p, 0, 16, s);
      cudaMemsetAsync(o.flags, 0, cbs[ui].size() * 4, s);
      launch_t1_encode(dv->work.as<bwc_float>(), dv->cbtab.as<CbDev>() + cb_base[ui],
                       (uint32_t)cbs[ui].size(), dv->sbtab.as<SbDev>(), o, max_cols, s,
                       dv->order.as<uint32_t>() + cb_base[ui], dv->queue.as<uint32_t>(), m2,
                       &mqt.t);
      unsigned long long cnt[2] = {0, 0};
      cudaMemcpyAsync(cnt, dv->symused.p, 16, cudaMemcpyDeviceToHost, s);
      if (!cuda_ok(cudaStreamSynchronize(s), "tier-1 encoding")) return 0;
      const unsigned long long used = cnt[0];
      if (used <= o.sym_cap) {
        dv->timings[8] += (double)cnt[1] * 1e-6;
        t_mq += mqt.total_ms();
        mq_launches += mqt.t.n;
        break;
      }
      if (attempt >= 3) {
        warn("o##########################################################o\n"
             "| ERROR: tier-1 symbol arena exhausted                     |\n"
             "o##########################################################o\n");
        return 0;
      }
      arena = used + (used >> 3) + (1 << 20);
    }
    cudaEventRecord(d2, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "compression kernels")) return 0;
    float x;
    cudaEventElapsedTime(&x, a, b2); t_norm += x;
    cudaEventElapsedTime(&x, b2, c2); t_dwt += x;
    cudaEventElapsedTime(&x, c2, d2); t_t1 += x;
    cudaEventElapsedTime(&x, c2, m2); t_model += x;
  }

  // tier-1 summary to the host
  cudaEventRecord(dv->ev[2], s);
  if (dv->device < 0 || dv->device >= 64) return 0;
  std::unique_lock<std::mutex> t1lock(g_t1host_mutex[dv->device]);
  T1Host h;
  h.layout(t1host_of(dv->device), ncb, ntiles, nu);
  uint8_t *const hK = h.K, *const hZ = h.Z;
  uint32_t *const hL = h.L, *const hflags = h.flags, *const hslopes = h.slopes;
  uint16_t *const hS = h.S;
  bwc_float *const hstats = h.stats;
  cudaMemcpyAsync(hK, dv->K.p, ncb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hZ, dv->Z.p, ncb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hL, dv->L.p, ncb * kMaxPasses * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hS, dv->S.p, ncb * (kMaxPasses + 1) * 2, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hflags, dv->flags.p, ncb * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hslopes, dv->slopes.p, 8 * ntiles, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hstats, dv->stats.p, 4 * sizeof(bwc_float) * nu, cudaMemcpyDeviceToHost, s);
  dwt_fault_download(h.fault, s);
  cudaEventRecord(dv->ev[3], s);
  if (!cuda_ok(cudaStreamSynchronize(s), "tier-1 download")) return 0;
  if (*h.fault) {
    warn("o##########################################################o\n"
         "| ERROR: the wavelet transform's input copies timed out    |\n"
         "o##########################################################o\n");
    return 0;
  }

  for (uint64_t i = 0; i < ncb; ++i) {
    if (hflags[i] & (1u | 16u)) {
      warn("o##########################################################o\n"
           "| ERROR: tier-1 output exceeded its codeblock buffer       |\n"
           "o##########################################################o\n");
      return 0;
    }
  }
  if (dv->dump_set) {
    const bwc_b200_stage_dump &d = dv->dump;
    const uint64_t n0 = cbs[0].size();
    if (d.K) std::memcpy(d.K, hK, n0);
    if (d.Z) std::memcpy(d.Z, hZ, n0);
    if (d.L) std::memcpy(d.L, hL, n0 * kMaxPasses * 4);
    if (d.S) std::memcpy(d.S, hS, n0 * (kMaxPasses + 1) * 2);
    if (d.flags) std::memcpy(d.flags, hflags, n0 * 4);
    if (d.stats) std::memcpy(d.stats, hstats, 4 * sizeof(bwc_float));
    if (d.bytes && d.byte_offsets) {
      uint64_t pos = 0;
      for (uint64_t i = 0; i < n0; ++i) {
        const uint64_t len = hZ[i] ? hL[i * kMaxPasses + hZ[i] - 1] : 0;
        d.byte_offsets[i] = pos;
        if (pos + len <= d.bytes_cap && len)
          cudaMemcpy(d.bytes + pos, dv->bytes.as<uint8_t>() + cbs[0][i].out_off, len,
                     cudaMemcpyDeviceToHost);
        pos += len;
      }
    }
  }
  for (size_t ui = 0; ui < nu; ++ui) {
    const TileUnit &u = units[ui];
    Parameter &par = eng->tiles[u.tile].params[u.param];
    par.pmin = hstats[4 * ui + 0];
    par.pmax = hstats[4 * ui + 1];
    par.alpha = hstats[4 * ui + 2];
    par.beta = hstats[4 * ui + 3];
    for (uint64_t i = 0; i < cbs[ui].size(); ++i) {
      const uint64_t g = cb_base[ui] + i;
      Codeblock &cb = par.codeblocks[i];
      CodedBlock &e = cb.enc;
      e.K = hK[g];
      e.Z = hZ[g];
      e.Kmsbs = e.K ? (uint8_t)(par.subbands[cb.subband].Kmax - e.K) : 0;
      for (int j = 0; j < e.Z; ++j) e.L[j] = hL[g * kMaxPasses + j];
      for (int j = 0; j <= e.Z; ++j) e.S[j] = hS[g * (kMaxPasses + 1) + j];
      cb.data_off = cbs[ui][i].out_off;
      cb.data_cap = cbs[ui][i].out_cap;
    }
  }
  for (size_t t = 0; t < ntiles; ++t) {
    eng->tiles[t].slope_min = (uint16_t)hslopes[2 * t];
    eng->tiles[t].slope_max = (uint16_t)hslopes[2 * t + 1];
  }
  t1lock.unlock();   // the tier-1 results are in the codec's own structures now

  // tier 2 on the host, tile by tile
  const auto h0 = std::chrono::steady_clock::now();
  for (Tile &tile : eng->tiles)
    if (t2_encode(codec, tile)) return 0;
  std::vector<uint8_t> blob;
  std::vector<GatherPiece> pieces;
  const uint64_t total = layout_codestream(codec, stream, blob, pieces);
  const auto h1 = std::chrono::steady_clock::now();
  if (!total) return 0;

  // codestream assembly on the device
  cudaEventRecord(dv->ev[4], s);
  if (!dv->blob.ensure(blob.size()) || !dv->pieces.ensure(pieces.size() * sizeof(GatherPiece)))
    return 0;
  cudaMemcpyAsync(dv->blob.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dv->pieces.p, pieces.data(), pieces.size() * sizeof(GatherPiece),
                  cudaMemcpyHostToDevice, s);
  const bool out_dev = is_device_pointer(stream->out);
  uint8_t *csdst;
  if (out_dev) {
    csdst = (uint8_t *)stream->out;
  } else {
    if (!dv->cs.ensure(total)) return 0;
    csdst = dv->cs.as<uint8_t>();
  }
  launch_gather(csdst, dv->blob.as<uint8_t>(), dv->bytes.as<uint8_t>(),
                dv->pieces.as<GatherPiece>(), pieces.size(), s);
  if (!out_dev) {
    HostStaging *hs = HostStaging::for_device(dv->device);
    if (!(hs && hs->download(stream->out, csdst, total, s)))
      cudaMemcpyAsync(stream->out, csdst, total, cudaMemcpyDeviceToHost, s);
  }
  cudaEventRecord(dv->ev[5], s);
  if (!cuda_ok(cudaStreamSynchronize(s), "codestream assembly")) return 0;

  float up = 0, dl = 0, as = 0;
  cudaEventElapsedTime(&up, dv->ev[0], dv->ev[1]);
  cudaEventElapsedTime(&dl, dv->ev[2], dv->ev[3]);
  cudaEventElapsedTime(&as, dv->ev[4], dv->ev[5]);
  dv->timings[0] = up;
  dv->timings[1] = t_norm;
  dv->timings[2] = t_dwt;
  dv->timings[3] = t_t1;
  dv->timings[4] = dl;
  dv->timings[5] = std::chrono::duration<double, std::milli>(h1 - h0).count();
  dv->timings[6] = as;
  dv->timings[7] = up + t_norm + t_dwt + t_t1 + dl + dv->timings[5] + as;
  dv->timings[9] = t_model;
  dv->timings[10] = t_mq;
  dv->timings[11] = mq_launches;
  dv->dump_set = false;
  return total;
}

// ---------------------------------------------------------------------------------------------
static uchar decompress_impl(bwc_codec *codec, bwc_stream *stream) {
  bwc_b200_engine *eng = codec->tile;
  if (!eng || eng->tiles.empty()) {
    warn(kCsError);
    return 1;
  }
  DeviceState *dv = device_state(codec);
  if (!dv) return 1;
  cudaStream_t s = dv->stream;
  bwc_gl_ctrl &c = codec->control;
  bwc_gl_inf &info = codec->info;
  const size_t dsz = (info.data_prec == bwc_precision_double) ? 8 : 4;
  const uint64_t out_bytes = info.nX * info.nY * info.nZ * info.nTS * (uint64_t)info.nPar * dsz;
  const uint64_t cs_len = c.codestreamSize;
  const std::vector<TileUnit> units = tile_units(codec);
  uint64_t nmax = 0;
  // Tiles that start past the first time step are written to time steps 0.. of the field (as
  // the reference's flush_buffer does): they overwrite earlier tiles there and leave later time
  // steps as they were in the caller's buffer, so that buffer is brought to the device first.
  bool keeps_output = false;
  for (const TileUnit &u : units) nmax = std::max(nmax, u.n);
  for (const Tile &t : eng->tiles) keeps_output |= t.box.TS0 != 0;

  cudaEventRecord(dv->ev[0], s);
  const uint8_t *dcs = (const uint8_t *)stream->inp;
  if (!is_device_pointer(stream->inp)) {
    if (!dv->cs.ensure(cs_len)) return 1;
    HostStaging *hs = HostStaging::for_device(dv->device);
    if (!(hs && hs->upload(dv->cs.p, stream->inp, cs_len, s)))
      cudaMemcpyAsync(dv->cs.p, stream->inp, cs_len, cudaMemcpyHostToDevice, s);
    dcs = dv->cs.as<uint8_t>();
  }
  const bool out_dev = is_device_pointer(stream->out);
  uint8_t *dout = (uint8_t *)stream->out;
  if (!out_dev) {
    if (!dv->outbuf.ensure(out_bytes)) return 1;
    dout = dv->outbuf.as<uint8_t>();
    if (keeps_output &&
        !cuda_ok(cudaMemcpyAsync(dout, stream->out, out_bytes, cudaMemcpyHostToDevice, s),
                 "output upload"))
      return 1;
  }
  cudaEventRecord(dv->ev[1], s);
  float t_t1 = 0, t_dwt = 0, t_norm = 0;
  for (size_t ui = 0; ui < units.size(); ++ui) {
    const TileUnit &u = units[ui];
    Parameter &par = eng->tiles[u.tile].params[u.param];
    const uint64_t n = u.n;
    const FieldDims &dims = u.dims;
    std::vector<CbDev> cbs;
    std::vector<SbDev> sbs;
    uint64_t bt, st;
    uint32_t mc;
    build_tables(par, dims, c.error_resilience, false, cbs, sbs, &bt, &st, &mc);
    const uint64_t ncb = cbs.size();
    std::vector<uint8_t> hK(ncb), hZ(ncb);
    std::vector<uint32_t> hLmax(ncb);
    std::vector<GatherPiece> pieces;
    uint64_t off = 0;
    for (uint64_t i = 0; i < ncb; ++i) {
      Codeblock &cb = par.codeblocks[i];
      const Subband &sb = par.subbands[cb.subband];
      hK[i] = (uint8_t)(sb.Kmax - cb.enc.Kmsbs);
      hZ[i] = cb.enc.Z;
      hLmax[i] = cb.enc.Z ? (uint32_t)cb.enc.L[cb.enc.Z - 1] : 0;
      cbs[i].out_off = off;
      uint64_t pos = off;
      for (auto &ch : cb.chunks) {
        if (ch.second) pieces.push_back({ch.first, pos, ch.second, 1});
        pos += ch.second;
      }
      off += ((std::max<uint64_t>(pos - off, hLmax[i]) + 16) + 15) & ~15ull;
    }
    const uint32_t state_cap = std::min<uint32_t>(mc, 6144);
    const size_t smem = 32 * 4 + (size_t)state_cap * 2 * 4;
    const bool big = mc > state_cap;
    uint64_t gstate_bytes = 0;
    if (big)
      for (uint64_t i = 0; i < ncb; ++i) gstate_bytes = std::max<uint64_t>(gstate_bytes, cbs[i].scratch_off);
    if (!dv->work.ensure(nmax * sizeof(bwc_float)) || !dv->temp.ensure(nmax * sizeof(bwc_float)) ||
        !dv->cbtab.ensure(sizeof(CbDev) * ncb) ||
        !dv->sbtab.ensure(sizeof(SbDev) * sbs.size()) || !dv->bytes.ensure(off + 64) ||
        !dv->mags.ensure(st * sizeof(bwc_raw)) || !dv->K.ensure(ncb) || !dv->Z.ensure(ncb) ||
        !dv->lmax.ensure(ncb * 4) || !dv->flags.ensure(ncb * 4) || !dv->counter.ensure(4) ||
        !dv->pieces.ensure(pieces.size() * sizeof(GatherPiece) + 16) ||
        !dv->order.ensure(ncb * 4) || (big && !dv->scratch.ensure(st * 2 + 64)))
      return 1;
    // decoding order: longest coded length first, so the longest decoding chains start first
    std::vector<uint32_t> dorder(ncb);
    for (uint64_t i = 0; i < ncb; ++i) dorder[i] = (uint32_t)i;
    std::stable_sort(dorder.begin(), dorder.end(),
                     [&](uint32_t a, uint32_t b) { return hLmax[a] > hLmax[b]; });
    cudaMemcpyAsync(dv->cbtab.p, cbs.data(), sizeof(CbDev) * ncb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->sbtab.p, sbs.data(), sizeof(SbDev) * sbs.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->K.p, hK.data(), ncb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->Z.p, hZ.data(), ncb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->lmax.p, hLmax.data(), ncb * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->order.p, dorder.data(), ncb * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dv->pieces.p, pieces.data(), pieces.size() * sizeof(GatherPiece),
                    cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(dv->bytes.p, 0, off + 64, s);
    cudaMemsetAsync(dv->flags.p, 0, ncb * 4, s);
    cudaMemsetAsync(dv->counter.p, 0, 4, s);
    launch_gather(dv->bytes.as<uint8_t>(), dcs, nullptr, dv->pieces.as<GatherPiece>(),
                  pieces.size(), s);
    const ScopedEvents evs;
    cudaEvent_t a = evs.e[0], b2 = evs.e[1], c2 = evs.e[2], d2 = evs.e[3];
    cudaEventRecord(a, s);
    cudaMemsetAsync(dv->temp.p, 0, n * sizeof(bwc_float), s);
    const int grid = t1_grid(nullptr, smem);
    launch_t1_decode_ex(dv->temp.as<bwc_float>(), dv->cbtab.as<CbDev>(), (uint32_t)ncb,
                        dv->sbtab.as<SbDev>(), dv->bytes.as<uint8_t>(), dv->K.as<uint8_t>(),
                        dv->Z.as<uint8_t>(), dv->lmax.as<uint32_t>(), c.error_resilience,
                        dv->mags.as<bwc_raw>(), dv->flags.as<uint32_t>(), state_cap,
                        big ? dv->scratch.as<uint16_t>() : nullptr, dv->counter.as<uint32_t>(),
                        grid, s, dv->order.as<uint32_t>(), mc);
    if (ui == 0 && dv->ddump_set && dv->ddump.dequantized)
      cudaMemcpyAsync(dv->ddump.dequantized, dv->temp.p, n * sizeof(bwc_float), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(b2, s);
    launch_dwt_inverse(dv->work.as<bwc_float>(), dv->temp.as<bwc_float>(), dims,
                       make_plan(c, par), s);
    if (ui == 0 && dv->ddump_set && dv->ddump.reconstructed)
      cudaMemcpyAsync(dv->ddump.reconstructed, dv->work.p, n * sizeof(bwc_float), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(c2, s);
    if (u.whole)
      launch_denormalize(dv->work.as<bwc_float>(), n, par.pmin, par.pmax, c.Qm,
                         dout + (uint64_t)u.param * n * dsz, dsz == 8, s);
    else
      launch_denormalize_box(dv->work.as<bwc_float>(), n, par.pmin, par.pmax, c.Qm, dout,
                             dsz == 8, u.map, s);
    cudaEventRecord(d2, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "decompression kernels")) return 1;
    float x;
    cudaEventElapsedTime(&x, a, b2); t_t1 += x;
    cudaEventElapsedTime(&x, b2, c2); t_dwt += x;
    cudaEventElapsedTime(&x, c2, d2); t_norm += x;
  }
  cudaEventRecord(dv->ev[2], s);
  if (!out_dev) {
    HostStaging *hs = HostStaging::for_device(dv->device);
    if (!(hs && hs->download(stream->out, dout, out_bytes, s)))
      cudaMemcpyAsync(stream->out, dout, out_bytes, cudaMemcpyDeviceToHost, s);
  }
  cudaEventRecord(dv->ev[3], s);
  if (!cuda_ok(cudaStreamSynchronize(s), "decompression download")) return 1;
  float up = 0, dl = 0;
  cudaEventElapsedTime(&up, dv->ev[0], dv->ev[1]);
  cudaEventElapsedTime(&dl, dv->ev[2], dv->ev[3]);
  dv->timings[0] = up;
  dv->timings[1] = t_norm;
  dv->timings[2] = t_dwt;
  dv->timings[3] = t_t1;
  dv->timings[4] = 0;
  dv->timings[5] = 0;
  dv->timings[6] = dl;
  dv->timings[7] = up + t_norm + t_dwt + t_t1 + dl;
  dv->ddump_set = false;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Batched compression: many independently configured codecs in one pass over the device.
//
// Every field keeps its own codec (geometry, rates, decomposition, input dtype), so its
// codestream is the one bwc_compress would write; only the execution changes:
//   * each (field, parameter) unit gets its own region of a batch working buffer; fill,
//     normalisation and the transform of the units run on several streams at once;
//   * tier-1 codes the codeblocks of ALL fields in one launch of each kernel (per field, tier-1
//     time is set by its longest codeblock, so separate calls would pay that chain per field);
//   * tier-2 runs for the fields in parallel host threads;
//   * one gather kernel assembles every codestream.
// One batch runs at a time per device (the batch buffers are shared); the call is serialised.
namespace {

struct BatchState {
  int device = -1;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t ev[6] = {};
  DevBuf in, work, temp, keys, stats, cbtab, sbtab, bytes, scratch, snaps, dmse, K, Z, L, S,
      flags, slopes, pcount, poff, symbols, symused, blob, pieces, cs, order, queue;
  double timings[8] = {};
  PinnedBuf t1host;   // page-locked home of the tier-1 results on the host
  // instantiated graphs of the fill/normalise/transform phase, by batch signature (geometry,
  // sources and buffer addresses); the few most recent are kept
  std::vector<std::pair<std::string, cudaGraphExec_t>> graphs;
  uint64_t graph_launches = 0, graph_captures = 0;
  // page-locked staging area for inputs in pageable host memory (kept, grown as needed)
  void *pinned = nullptr;
  uint64_t pinned_cap = 0;
};

constexpr int kBatchStreams = 8;
std::mutex g_batch_mutex;
BatchState *g_batch[64] = {};

BatchState *batch_state() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!g_batch[dev]) {
    BatchState *b = new (std::nothrow) BatchState();
    if (!b) return nullptr;
    b->device = dev;
    if (!cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream")) {
      delete b;
      return nullptr;
    }
    b->side.resize(kBatchStreams);
    b->join.resize(kBatchStreams + 1);
    for (auto &x : b->side) cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
    for (auto &e : b->join) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto &e : b->ev) cudaEventCreate(&e);
    g_batch[dev] = b;
  }
  return g_batch[dev];
}

struct BatchUnit {
  uint32_t field;
  uint32_t tile;       // tile index within the field
  int param;
  uint64_t n;          // values
  BoxMap map;          // the tile's samples in the field's input
  bool whole;          // the field is one tile (its parameter is contiguous)
  uint64_t work_off;   // element offset in the batch working buffers
  const uint8_t *src;  // device address of the unit's input values
  bool src_double;
  FieldDims dims;
  DwtPlan plan;
  uint8_t Qm;
  uint64_t cb_first, cb_count;
};

}  // namespace

static uchar compress_batch_impl(bwc_codec *const *codecs, bwc_stream *const *streams,
                                 uint32_t nf, size_t *sizes) {
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  BatchState *bs = batch_state();
  if (!bs) return 1;
  cudaStream_t s = bs->stream;
  for (uint32_t i = 0; i < nf; ++i) {
    sizes[i] = 0;
    if (!codecs[i] || !streams[i] || !codecs[i]->tile || codecs[i]->tile->tiles.empty()) {
      warn("o##########################################################o\n"
           "| ERROR: bwc_create_compression has not been called        |\n"
           "o##########################################################o\n");
      return 1;
    }
  }
  cudaEventRecord(bs->ev[0], s);
  // ---- units, inputs, tables
  std::vector<BatchUnit> units;
  std::vector<uint64_t> in_off(nf, ~0ull), in_bytes(nf, 0);
  uint64_t work_total = 0, in_total = 0;
  // slope-range slot of every (field, tile): tile t of field i uses slot tile_base[i] + t
  std::vector<uint32_t> tile_base(nf + 1, 0);
  for (uint32_t i = 0; i < nf; ++i) {
    bwc_codec *codec = codecs[i];
    const bwc_gl_inf &info = codec->info;
    const size_t dsz = (info.data_prec == bwc_precision_double) ? 8 : 4;
    in_bytes[i] = info.nX * info.nY * info.nZ * info.nTS * (uint64_t)info.nPar * dsz;
    if (!is_device_pointer(streams[i]->inp)) {
      in_off[i] = in_total;
      in_total += (in_bytes[i] + 255) & ~255ull;
    }
    tile_base[i + 1] = tile_base[i] + (uint32_t)codec->tile->tiles.size();
    for (const TileUnit &tu : tile_units(codec)) {
      const Tile &tile = codec->tile->tiles[tu.tile];
      BatchUnit u{};
      u.field = i;
      u.tile = tu.tile;
      u.param = (int)tu.param;
      u.n = tu.n;
      u.map = tu.map;
      u.whole = tu.whole;
      u.work_off = work_total;
      work_total += (u.n + 31) & ~31ull;
      u.src_double = dsz == 8;
      u.dims = tu.dims;
      u.plan = make_plan(codec->control, tile.params[tu.param]);
      u.Qm = codec->control.Qm;
      units.push_back(u);
    }
  }
  const uint32_t nslots = tile_base[nf];
  std::vector<CbDev> allcb;
  std::vector<SbDev> allsb;
  uint64_t bytes_total = 0, scratch_total = 0, total_samples = 0;
  uint32_t max_cols = 0;
  for (BatchUnit &u : units) {
    Tile &tile = codecs[u.field]->tile->tiles[u.tile];
    std::vector<CbDev> cbs;
    std::vector<SbDev> sbs;
    uint64_t bt, st;
    uint32_t mc;
    build_tables(tile.params[u.param], u.dims, codecs[u.field]->control.error_resilience, true,
                 cbs, sbs, &bt, &st, &mc);
    max_cols = std::max(max_cols, mc);
    u.cb_first = allcb.size();
    u.cb_count = cbs.size();
    for (CbDev &d : cbs) {
      d.base = u.work_off;
      d.out_off += bytes_total;
      d.scratch_off += scratch_total;
      d.sb += (uint32_t)allsb.size();
      d.slot = tile_base[u.field] + u.tile;
      total_samples += (uint64_t)d.w * ((d.h + 3) / 4) * 4 * d.d * d.nt;
      allcb.push_back(d);
    }
    allsb.insert(allsb.end(), sbs.begin(), sbs.end());
    bytes_total += bt;
    scratch_total += st;
  }
  const uint64_t ncb = allcb.size(), nu = units.size();
  if (t1_model_smem(max_cols) > 200 * 1024) {
    warn("o##########################################################o\n"
         "| ERROR: codeblocks above 2^18 samples are not supported   |\n"
         "o##########################################################o\n");
    return 1;
  }
  if (!bs->in.ensure(in_total) || !bs->work.ensure(work_total * sizeof(bwc_float)) ||
      !bs->temp.ensure(work_total * sizeof(bwc_float)) || !bs->keys.ensure(16 * nu) ||
      !bs->stats.ensure(4 * sizeof(bwc_float) * nu) || !bs->cbtab.ensure(sizeof(CbDev) * ncb) ||
      !bs->sbtab.ensure(sizeof(SbDev) * allsb.size()) || !bs->bytes.ensure(bytes_total) ||
      !bs->scratch.ensure(scratch_total) || !bs->snaps.ensure(ncb * kMaxPasses * 16) ||
      !bs->dmse.ensure(ncb * kMaxPasses * 8) || !bs->K.ensure(ncb) || !bs->Z.ensure(ncb) ||
      !bs->L.ensure(ncb * kMaxPasses * 4) || !bs->S.ensure(ncb * (kMaxPasses + 1) * 2) ||
      !bs->flags.ensure(ncb * 4) || !bs->slopes.ensure(8 * nslots) ||
      !bs->pcount.ensure(ncb * kMaxPasses * 4) || !bs->poff.ensure(ncb * kMaxPasses * 8) ||
      !bs->symused.ensure(16) || !bs->order.ensure(ncb * 4) || !bs->queue.ensure(32))
    return 1;
  const std::vector<uint32_t> order = work_order(allcb, allsb, 0, ncb);
  // Inputs in pageable host memory go through a page-locked staging area: several host threads
  // copy them in, then each is uploaded by DMA (a copy straight from pageable memory is staged
  // by the driver in small page-locked chunks, several times slower).  Page-locked host inputs
  // are uploaded as they are; device inputs need no upload.
  std::vector<uint64_t> stage_off(nf, ~0ull);
  uint64_t stage_total = 0;
  for (uint32_t i = 0; i < nf; ++i)
    if (in_off[i] != ~0ull && !is_pinned_host(streams[i]->inp)) {
      stage_off[i] = stage_total;
      stage_total += in_bytes[i];
    }
  if (stage_total > bs->pinned_cap) {
    if (bs->pinned) cudaFreeHost(bs->pinned);
    bs->pinned = nullptr;
    bs->pinned_cap = 0;
    if (cudaHostAlloc(&bs->pinned, stage_total, cudaHostAllocDefault) == cudaSuccess) {
      bs->pinned_cap = stage_total;
    } else {
      cudaGetLastError();   // no staging area: upload from pageable memory directly
      bs->pinned = nullptr;
    }
  }
  const bool staged = stage_total > 0 && bs->pinned != nullptr;
  if (staged) {
    // an earlier call that returned early may still be uploading from the staging area
    if (!cuda_ok(cudaStreamSynchronize(s), "batch staging")) return 1;
    // the inputs, concatenated, cut into equal spans, one per thread
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned k = 0; k < nt; ++k)
      th.emplace_back([&, k] {
        const uint64_t a = stage_total * k / nt, b = stage_total * (k + 1) / nt;
        for (uint32_t i = 0; i < nf; ++i) {
          if (stage_off[i] == ~0ull) continue;
          const uint64_t lo = std::max(a, stage_off[i]);
          const uint64_t hi = std::min(b, stage_off[i] + in_bytes[i]);
          if (lo < hi)
            std::memcpy(static_cast<uint8_t *>(bs->pinned) + lo,
                        static_cast<const uint8_t *>(streams[i]->inp) + (lo - stage_off[i]),
                        hi - lo);
        }
      });
    for (auto &t : th) t.join();
  }
  for (uint32_t i = 0; i < nf; ++i)
    if (in_off[i] != ~0ull) {
      const void *from = (staged && stage_off[i] != ~0ull)
                             ? static_cast<const void *>(static_cast<uint8_t *>(bs->pinned) + stage_off[i])
                             : streams[i]->inp;
      cudaMemcpyAsync(bs->in.as<uint8_t>() + in_off[i], from, in_bytes[i],
                      cudaMemcpyHostToDevice, s);
    }
  for (BatchUnit &u : units) {
    const bwc_codec *codec = codecs[u.field];
    const size_t dsz = u.src_double ? 8 : 4;
    const uint8_t *base = (in_off[u.field] != ~0ull) ? bs->in.as<uint8_t>() + in_off[u.field]
                                                     : (const uint8_t *)streams[u.field]->inp;
    u.src = u.whole ? base + (uint64_t)u.param * u.n * dsz : base;
    (void)codec;
  }
  cudaMemcpyAsync(bs->cbtab.p, allcb.data(), sizeof(CbDev) * ncb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(bs->sbtab.p, allsb.data(), sizeof(SbDev) * allsb.size(), cudaMemcpyHostToDevice,
                  s);
  cudaMemcpyAsync(bs->order.p, order.data(), ncb * 4, cudaMemcpyHostToDevice, s);
  {
    std::vector<uint32_t> init(2 * nslots);
    for (uint32_t i = 0; i < nslots; ++i) {
      init[2 * i] = 0xFFFF;
      init[2 * i + 1] = 0;
    }
    cudaMemcpyAsync(bs->slopes.p, init.data(), 8 * nslots, cudaMemcpyHostToDevice, s);
    std::vector<uint64_t> keys(2 * nu);
    for (uint64_t u = 0; u < nu; ++u) {
      keys[2 * u] = ~0ull;
      keys[2 * u + 1] = 0;
    }
    cudaMemcpyAsync(bs->keys.p, keys.data(), 16 * nu, cudaMemcpyHostToDevice, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "batch set-up")) return 1;   // host vectors die here
  }
  cudaEventRecord(bs->ev[1], s);

  // ---- fill, normalise and transform every unit, spread over the side streams: captured once
  // into a CUDA graph per batch signature and replayed
  auto enqueue_transforms = [&]() {
    cudaEventRecord(bs->join[kBatchStreams], s);
    for (int k = 0; k < kBatchStreams; ++k)
      cudaStreamWaitEvent(bs->side[k], bs->join[kBatchStreams], 0);
    for (uint64_t ui = 0; ui < nu; ++ui) {
      const BatchUnit &u = units[ui];
      cudaStream_t ss = bs->side[ui % kBatchStreams];
      bwc_float *temp = bs->temp.as<bwc_float>() + u.work_off;
      bwc_float *work = bs->work.as<bwc_float>() + u.work_off;
      if (u.whole)
        launch_fill_minmax(u.src, u.src_double, u.n, temp, bs->keys.as<uint64_t>() + 2 * ui, ss);
      else
        launch_fill_minmax_box(u.src, u.src_double, u.n, u.map, temp,
                               bs->keys.as<uint64_t>() + 2 * ui, ss);
      launch_normalize(temp, u.n, bs->keys.as<uint64_t>() + 2 * ui, u.Qm,
                       bs->stats.as<bwc_float>() + 4 * ui, ss);
      launch_dwt_forward(work, temp, u.dims, u.plan, ss);
    }
    for (int k = 0; k < kBatchStreams; ++k) {
      cudaEventRecord(bs->join[k], bs->side[k]);
      cudaStreamWaitEvent(s, bs->join[k], 0);
    }
  };
  std::string sig;
  {
    char buf[160];
    snprintf(buf, sizeof buf, "%p %p %p %p|", bs->work.p, bs->temp.p, bs->keys.p, bs->stats.p);
    sig = buf;
    for (const BatchUnit &u : units) {
      snprintf(buf, sizeof buf, "%p %d %llu %llu %llu %llu %llu %d %u|", (const void *)u.src,
               (int)u.src_double, (unsigned long long)u.n, (unsigned long long)u.work_off,
               (unsigned long long)u.dims.width, (unsigned long long)u.dims.height,
               (unsigned long long)(u.dims.depth * 65536 + u.dims.dt), u.plan.levels, u.Qm);
      sig += buf;
      if (!u.whole) {
        snprintf(buf, sizeof buf, "b%llu %llu %llu %llu|", (unsigned long long)u.map.base,
                 (unsigned long long)u.map.sy, (unsigned long long)u.map.sz,
                 (unsigned long long)u.map.st);
        sig += buf;
      }
      for (int k = 0; k < 4; ++k) sig += std::to_string(u.plan.kern[k]);
      for (int l = 0; l < u.plan.levels; ++l)
        sig += std::to_string(u.plan.axis_on[l] | (u.plan.odd[l] << 8)) + ",";
    }
  }
  cudaGraphExec_t exec = nullptr;
  for (auto &g : bs->graphs)
    if (g.first == sig) exec = g.second;
  if (!exec) {
    cudaGraph_t graph = nullptr;
    dwt_setup();
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      enqueue_transforms();
      if (cudaStreamEndCapture(s, &graph) == cudaSuccess && graph &&
          cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        bs->graphs.emplace_back(sig, exec);
        ++bs->graph_captures;
        if (bs->graphs.size() > 8) {
          cudaGraphExecDestroy(bs->graphs.front().second);
          bs->graphs.erase(bs->graphs.begin());
        }
      } else {
        exec = nullptr;
      }
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();
  }
  if (exec) {
    if (!cuda_ok(cudaGraphLaunch(exec, s), "batch transform graph")) return 1;
    ++bs->graph_launches;
  } else {
    enqueue_transforms();   // capture unavailable: the same launches, directly
  }
  cudaEventRecord(bs->ev[2], s);

  // ---- tier-1 over all codeblocks (grown and repeated if the symbol arena was too small)
  uint64_t arena = std::max<uint64_t>(1 << 20, total_samples * (kPrecBit + 1) * 9 / 8);
  T1EncOut o;
  o.bytes = bs->bytes.as<uint8_t>();
  o.K = bs->K.as<uint8_t>();
  o.Z = bs->Z.as<uint8_t>();
  o.L = bs->L.as<uint32_t>();
  o.S = bs->S.as<uint16_t>();
  o.slopes = bs->slopes.as<uint32_t>();
  o.flags = bs->flags.as<uint32_t>();
  o.planes = bs->scratch.as<uint8_t>();
  o.snaps = bs->snaps.as<uint64_t>();
  o.dmse = bs->dmse.as<int64_t>();
  o.pass_count = bs->pcount.as<uint32_t>();
  o.pass_off = bs->poff.as<uint64_t>();
  o.sym_used = bs->symused.as<unsigned long long>();
  for (int attempt = 0;; ++attempt) {
    if (!bs->symbols.ensure(arena + 256)) return 1;
    o.symbols = bs->symbols.as<uint8_t>();
    o.sym_cap = bs->symbols.cap - 256;
    cudaMemsetAsync(bs->symused.p, 0, 16, s);
    cudaMemsetAsync(bs->flags.p, 0, ncb * 4, s);
    launch_t1_encode(bs->work.as<bwc_float>(), bs->cbtab.as<CbDev>(), (uint32_t)ncb,
                     bs->sbtab.as<SbDev>(), o, max_cols, s, bs->order.as<uint32_t>(),
                     bs->queue.as<uint32_t>());
    unsigned long long used = 0;
    cudaMemcpyAsync(&used, bs->symused.p, 8, cudaMemcpyDeviceToHost, s);
    if (!cuda_ok(cudaStreamSynchronize(s), "batch tier-1 encoding")) return 1;
    if (used <= o.sym_cap) break;
    if (attempt >= 3) {
      warn("o##########################################################o\n"
           "| ERROR: tier-1 symbol arena exhausted                     |\n"
           "o##########################################################o\n");
      return 1;
    }
    arena = used + (used >> 3) + (1 << 20);
  }
  cudaEventRecord(bs->ev[3], s);
  T1Host h;
  h.layout(bs->t1host, ncb, nslots, nu);
  uint8_t *const hK = h.K, *const hZ = h.Z;
  uint32_t *const hL = h.L, *const hflags = h.flags, *const hslopes = h.slopes;
  uint16_t *const hS = h.S;
  bwc_float *const hstats = h.stats;
  cudaMemcpyAsync(hK, bs->K.p, ncb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hZ, bs->Z.p, ncb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hL, bs->L.p, ncb * kMaxPasses * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hS, bs->S.p, ncb * (kMaxPasses + 1) * 2, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hflags, bs->flags.p, ncb * 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hslopes, bs->slopes.p, 8 * nslots, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hstats, bs->stats.p, 4 * sizeof(bwc_float) * nu, cudaMemcpyDeviceToHost, s);
  dwt_fault_download(h.fault, s);
  if (!cuda_ok(cudaStreamSynchronize(s), "batch tier-1 download")) return 1;
  if (*h.fault) {
    warn("o##########################################################o\n"
         "| ERROR: the wavelet transform's input copies timed out    |\n"
         "o##########################################################o\n");
    return 1;
  }
  for (uint64_t c = 0; c < ncb; ++c)
    if (hflags[c] & (1u | 16u)) {
      warn("o##########################################################o\n"
           "| ERROR: tier-1 output exceeded its codeblock buffer       |\n"
           "o##########################################################o\n");
      return 1;
    }
  const auto h0 = std::chrono::steady_clock::now();

  // ---- tier-2 and layout per field, in parallel host threads
  std::vector<std::vector<uint8_t>> blobs(nf);
  std::vector<std::vector<GatherPiece>> fpieces(nf);
  std::vector<uint64_t> totals(nf, 0);
  std::vector<uint64_t> first_unit(nf + 1, 0);
  for (uint64_t ui = 0; ui < nu; ++ui) first_unit[units[ui].field + 1] = ui + 1;
  for (uint32_t i = 0; i < nf; ++i) first_unit[i + 1] = std::max(first_unit[i + 1], first_unit[i]);
  std::atomic<uint32_t> next{0};
  std::atomic<int> failed{0};
  auto worker = [&]() {
    t_rate_control_in_parallel_fields = nf > 1;   // a lone field may spread its probes
    for (;;) {
      const uint32_t i = next.fetch_add(1);
      if (i >= nf) return;
      bwc_codec *codec = codecs[i];
      for (uint64_t ui = first_unit[i]; ui < first_unit[i + 1]; ++ui) {
        const BatchUnit &u = units[ui];
        Parameter &par = codec->tile->tiles[u.tile].params[u.param];
        par.pmin = hstats[4 * ui + 0];
        par.pmax = hstats[4 * ui + 1];
        par.alpha = hstats[4 * ui + 2];
        par.beta = hstats[4 * ui + 3];
        for (uint64_t j = 0; j < u.cb_count; ++j) {
          const uint64_t g = u.cb_first + j;
          Codeblock &cb = par.codeblocks[j];
          CodedBlock &e = cb.enc;
          e.K = hK[g];
          e.Z = hZ[g];
          e.Kmsbs = e.K ? (uint8_t)(par.subbands[cb.subband].Kmax - e.K) : 0;
          for (int z = 0; z < e.Z; ++z) e.L[z] = hL[g * kMaxPasses + z];
          for (int z = 0; z <= e.Z; ++z) e.S[z] = hS[g * (kMaxPasses + 1) + z];
          cb.data_off = allcb[g].out_off;
          cb.data_cap = allcb[g].out_cap;
        }
      }
      bool ok = true;
      for (Tile &tile : codec->tile->tiles) {
        tile.slope_min = (uint16_t)hslopes[2 * (tile_base[i] + tile.index)];
        tile.slope_max = (uint16_t)hslopes[2 * (tile_base[i] + tile.index) + 1];
        if (t2_encode(codec, tile)) {
          ok = false;
          break;
        }
      }
      if (!ok) {
        failed = 1;
        continue;
      }
      totals[i] = layout_codestream(codec, streams[i], blobs[i], fpieces[i]);
      if (!totals[i]) failed = 1;
    }
  };
  {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>(hw, nf);
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    t_rate_control_in_parallel_fields = false;
    for (auto &t : pool) t.join();
  }
  if (failed) return 1;
  const auto h1 = std::chrono::steady_clock::now();

  // ---- one gather for every codestream, then each to its stream->out
  std::vector<uint8_t> blob;
  std::vector<GatherPiece> pieces;
  std::vector<uint64_t> cs_off(nf);
  uint64_t cs_total = 0;
  for (uint32_t i = 0; i < nf; ++i) {
    const uint64_t boff = blob.size();
    blob.insert(blob.end(), blobs[i].begin(), blobs[i].end());
    cs_off[i] = cs_total;
    for (GatherPiece pc : fpieces[i]) {
      if (pc.from_blob) pc.src += boff;
      pc.dst += cs_off[i];
      pieces.push_back(pc);
    }
    cs_total += (totals[i] + 255) & ~255ull;
  }
  cudaEventRecord(bs->ev[4], s);
  if (!bs->blob.ensure(blob.size()) || !bs->pieces.ensure(pieces.size() * sizeof(GatherPiece)) ||
      !bs->cs.ensure(cs_total))
    return 1;
  cudaMemcpyAsync(bs->blob.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(bs->pieces.p, pieces.data(), pieces.size() * sizeof(GatherPiece),
                  cudaMemcpyHostToDevice, s);
  launch_gather(bs->cs.as<uint8_t>(), bs->blob.as<uint8_t>(), bs->bytes.as<uint8_t>(),
                bs->pieces.as<GatherPiece>(), pieces.size(), s);
  for (uint32_t i = 0; i < nf; ++i) {
    const bool out_dev = is_device_pointer(streams[i]->out);
    cudaMemcpyAsync(streams[i]->out, bs->cs.as<uint8_t>() + cs_off[i], totals[i],
                    out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
  }
  cudaEventRecord(bs->ev[5], s);
  if (!cuda_ok(cudaStreamSynchronize(s), "batch codestream assembly")) return 1;
  float t[5] = {0, 0, 0, 0, 0};
  cudaEventElapsedTime(&t[0], bs->ev[0], bs->ev[1]);
  cudaEventElapsedTime(&t[1], bs->ev[1], bs->ev[2]);
  cudaEventElapsedTime(&t[2], bs->ev[2], bs->ev[3]);
  cudaEventElapsedTime(&t[3], bs->ev[4], bs->ev[5]);
  bs->timings[0] = t[0];   // set-up and uploads
  bs->timings[1] = t[1];   // fill, normalise, transform
  bs->timings[2] = t[2];   // tier-1
  bs->timings[3] = std::chrono::duration<double, std::milli>(h1 - h0).count();   // tier-2
  bs->timings[4] = t[3];   // gather and outputs
  cudaEventElapsedTime(&t[4], bs->ev[0], bs->ev[5]);
  bs->timings[5] = t[4];   // whole call
  for (uint32_t i = 0; i < nf; ++i) sizes[i] = totals[i];
  return 0;
}

}  // namespace bwcb

using namespace bwcb;

extern "C" size_t bwc_compress(bwc_codec *const codec, bwc_stream *const data) {
  if (!codec || !data) return 0;
  return guarded<size_t>(0, [&] { return compress_impl(codec, data); });
}

extern "C" uchar bwc_decompress(bwc_codec *const codec, bwc_stream *const stream) {
  if (!codec || !stream) return 1;
  return guarded<uchar>(1, [&] { return decompress_impl(codec, stream); });
}

extern "C" int bwc_b200_precision_bits(void) { return kPrecBit; }

extern "C" void bwc_b200_reset_gain_state(void) { reset_gain_lut(); }

extern "C" void bwc_b200_get_gain_state(double *out30) { copy_gain_lut(out30); }

extern "C" uint64 bwc_b200_num_codeblocks(bwc_codec *const codec, uint8 const param) {
  if (!codec || !codec->tile || codec->tile->tiles.empty()) return 0;
  if (param >= codec->tile->tiles[0].params.size()) return 0;
  return codec->tile->tiles[0].params[param].codeblocks.size();
}

extern "C" void bwc_b200_set_stage_dump(bwc_codec *const codec, bwc_b200_stage_dump const *dump) {
  DeviceState *d = device_state(codec);
  if (!d) return;
  d->dump_set = dump != nullptr;
  if (dump) d->dump = *dump;
}

extern "C" void bwc_b200_set_decode_dump(bwc_codec *const codec, bwc_b200_decode_dump const *dump) {
  DeviceState *d = device_state(codec);
  if (!d) return;
  d->ddump_set = dump != nullptr;
  if (dump) d->ddump = *dump;
}

extern "C" int bwc_b200_last_timings(bwc_codec *const codec, double *out_ms, int n) {
  if (!codec || !codec->tile || !codec->tile->dev) return 0;
  const int k = std::min(n, 12);
  for (int i = 0; i < k; ++i) out_ms[i] = codec->tile->dev->timings[i];
  return k;
}

extern "C" uchar bwc_b200_compress_batch(bwc_codec *const *codecs, bwc_stream *const *streams,
                                         uint32 n, size_t *sizes) {
  if (!codecs || !streams || !sizes || n == 0) return 1;
  return guarded<uchar>(1, [&] { return compress_batch_impl(codecs, streams, n, sizes); });
}

extern "C" int bwc_b200_last_batch_timings(double *out_ms, int n) {
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || !g_batch[dev]) return 0;
  const int k = std::min(n, 8);
  g_batch[dev]->timings[6] = (double)g_batch[dev]->graph_captures;
  g_batch[dev]->timings[7] = (double)g_batch[dev]->graph_launches;
  for (int i = 0; i < k; ++i) out_ms[i] = g_batch[dev]->timings[i];
  return k;
}
