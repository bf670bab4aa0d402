// Tier-1 encoding of one codeblock with no memory allocation at all:
// bwc_b200_t1_encode_codeblock_static.
//
// Who needs it: code that must not call cudaMalloc -- a caller working inside a framework whose
// memory pool owns the device memory, or a latency-bound service that cannot afford the implicit
// synchronisation of an allocation.  Such a caller owns its inputs and outputs already; what it
// cannot provide is this library's tier-1 working memory (bit planes, the symbol arena, coder
// snapshots).  Here that working memory is one fixed static device array, sized for the largest
// codeblock the entry point accepts; every GPU that loads the library holds it until the
// process exits.
//
// The kernels are the ones bwc_compress runs (t1_model_kernel, t1_mq_kernel through
// launch_t1_encode); only where their scratch lives differs.  The codeblock and subband records
// reach the static area through a one-thread set-up kernel that takes them as arguments, so no
// host memory is read after the call returns.
#include <cstdio>
#include <mutex>

#include "bwc_b200.h"
#include "device_common.cuh"

namespace bwcb {
namespace {

// Largest codeblock: 4096 stripe columns (16384 samples, e.g. 32 x 32 x 16 -- the codeblock of
// the benchmark workload -- or 64 x 64 x 4).
constexpr uint32_t kStaticMaxCols = 4096;
constexpr uint64_t kMaxPlanes = kPrecBit + 1;
// A stripe column emits at most 10 symbols per bit plane (run mode: 3, then sign and three
// significance/sign pairs), error resilience 4 per plane, every pass is padded to 16 bytes, and
// the MQ coder reads up to 256 bytes past the last chunk.
constexpr uint64_t kArenaBytes =
    ((uint64_t)kStaticMaxCols * 10 * kMaxPlanes + 4 * kMaxPlanes + 16ull * kMaxPasses + 256 +
     255) & ~255ull;

constexpr uint64_t round256(uint64_t v) { return (v + 255) & ~255ull; }
// layout of the static area
constexpr uint64_t kOffPlanes = 0;
constexpr uint64_t kOffArena = round256(kOffPlanes + (uint64_t)kStaticMaxCols * kMaxPlanes);
constexpr uint64_t kOffSnaps = round256(kOffArena + kArenaBytes);
constexpr uint64_t kOffDmse = round256(kOffSnaps + 16ull * kMaxPasses);
constexpr uint64_t kOffPcount = round256(kOffDmse + 8ull * kMaxPasses);
constexpr uint64_t kOffPoff = round256(kOffPcount + 4ull * kMaxPasses);
constexpr uint64_t kOffUsed = round256(kOffPoff + 8ull * kMaxPasses);   // arena bump counter,
                                                                         // decisions coded
constexpr uint64_t kOffSlopes = kOffUsed + 16;                           // slope min / max
constexpr uint64_t kOffFlags = kOffSlopes + 8;                           // codeblock flags
constexpr uint64_t kOffCb = round256(kOffFlags + 4);
constexpr uint64_t kOffSb = round256(kOffCb + sizeof(CbDev));
constexpr uint64_t kStaticBytes = round256(kOffSb + sizeof(SbDev));

// about 2.9 MB in the double build, 1.5 MB in the single build
static __device__ __align__(256) unsigned char g_t1_static[kStaticBytes];

// device address of g_t1_static, looked up once per device (in host code the array's name is
// only a host-side stand-in for the symbol)
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_static_addr[kMaxDevices] = {};

unsigned char *static_area(int device) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_static_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_t1_static);
    if (e != cudaSuccess) {
      fprintf(stderr, "bwc: static tier-1 scratch unavailable on device %d: %s\n", device,
              cudaGetErrorString(e));
      return nullptr;
    }
    g_static_addr[device] = static_cast<unsigned char *>(p);
  }
  return g_static_addr[device];
}

// Writes the call's codeblock and subband records into the static area and clears what must
// start from zero: the symbol bump counter, the flags and the slope range (minimum 0xFFFF).
// Planes, symbol chunks, snapshots and per-pass records are rewritten before they are read.
__global__ void static_setup_kernel(unsigned char *base, CbDev cb, SbDev sb) {
  *reinterpret_cast<CbDev *>(base + kOffCb) = cb;
  *reinterpret_cast<SbDev *>(base + kOffSb) = sb;
  reinterpret_cast<unsigned long long *>(base + kOffUsed)[0] = 0ull;
  reinterpret_cast<unsigned long long *>(base + kOffUsed)[1] = 0ull;
  uint32_t *slopes = reinterpret_cast<uint32_t *>(base + kOffSlopes);
  slopes[0] = 0xFFFF;
  slopes[1] = 0;
  *reinterpret_cast<uint32_t *>(base + kOffFlags) = 0;
}

// Copies the codeblock's flags to the caller's status word (device to device, no host copy).
__global__ void static_status_kernel(const unsigned char *base, uint32_t *status) {
  *status = *reinterpret_cast<const uint32_t *>(base + kOffFlags);
}

int reject(const char *why) {
  fprintf(stderr, "bwc_b200_t1_encode_codeblock_static: %s\n", why);
  return 1;
}

}  // namespace
}  // namespace bwcb

using namespace bwcb;

extern "C" int bwc_b200_t1_encode_codeblock_static(
    const bwc_float *coeffs, uint64 nX, uint64 nY, uint64 nZ, uint64 nTS, const uint64 *box,
    bwc_float qt_eff, double gain_step2, uint8 highband, uchar erres, uint8 *K, uint8 *Z,
    uint32 *L, uint16 *S, uint8 *bytes, uint32 bytes_cap, uint32 *status, void *stream) {
  if (!coeffs || !box || !K || !Z || !L || !S || !bytes || !status)
    return reject("a buffer pointer is NULL");
  if (!nX || !nY || !nZ || !nTS) return reject("field extents must be positive");
  const uint64 dims[4] = {nX, nY, nZ, nTS};
  for (int a = 0; a < 4; ++a)
    if (box[a] >= box[4 + a] || box[4 + a] > dims[a])
      return reject("codeblock box is empty or outside the field");
  const uint64 w = box[4] - box[0], h = box[5] - box[1], d = box[6] - box[2], nt = box[7] - box[3];
  const uint64 ncols = w * ((h + 3) / 4) * d * nt;
  if (ncols > kStaticMaxCols) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "codeblock has %llu stripe columns; the static working memory holds at most %u "
             "(16384 samples)", (unsigned long long)ncols, kStaticMaxCols);
    return reject(msg);
  }
  // An error left pending by the caller's own earlier CUDA calls would be reported after the
  // launches below as if they had failed; refuse before queuing anything instead.
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "a CUDA error is pending from earlier calls (%s); nothing queued",
             cudaGetErrorString(pending));
    return reject(msg);
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return reject("no usable current CUDA device");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s) {
    // the static area's address is the current device's: the stream must belong to it
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) return reject("invalid stream");
    if (sdev != device) return reject("the stream belongs to another device than the current one");
  }
  unsigned char *base = static_area(device);
  if (!base) return 1;

  CbDev cb{};
  cb.x0 = (uint32_t)box[0];
  cb.y0 = (uint32_t)box[1];
  cb.z0 = (uint32_t)box[2];
  cb.t0 = (uint32_t)box[3];
  cb.w = (uint32_t)w;
  cb.h = (uint32_t)h;
  cb.d = (uint32_t)d;
  cb.nt = (uint32_t)nt;
  cb.out_off = 0;
  cb.scratch_off = 0;
  cb.out_cap = bytes_cap;
  cb.sb = 0;
  cb.base = 0;
  cb.sy = nX;
  cb.sz = nX * nY;
  cb.st = nX * nY * nZ;
  cb.slot = 0;
  SbDev sb{};
  sb.gain_step2 = gain_step2;
  sb.qt_eff = qt_eff;
  sb.Kmax = 0;
  // significance-context class from the subband's high-pass axes (tier1.c:2416-2446)
  sb.cls = ((highband & 3) == 1) ? 1u : ((highband & 3) == 3) ? 2u : 0u;
  sb.erres = erres ? 1u : 0u;

  // The static area keeps the previous call's contents; the set-up kernel writes this call's
  // records and clears the counters before the tier-1 kernels run on the same stream.
  static_setup_kernel<<<1, 1, 0, s>>>(base, cb, sb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "bwc_b200_t1_encode_codeblock_static: set-up launch: %s\n",
            cudaGetErrorString(e));
    return 1;
  }

  T1EncOut o;
  o.bytes = bytes;
  o.K = K;
  o.Z = Z;
  o.L = L;
  o.S = S;
  o.slopes = reinterpret_cast<uint32_t *>(base + kOffSlopes);
  o.flags = reinterpret_cast<uint32_t *>(base + kOffFlags);
  o.planes = base + kOffPlanes;
  o.snaps = reinterpret_cast<uint64_t *>(base + kOffSnaps);
  o.dmse = reinterpret_cast<int64_t *>(base + kOffDmse);
  o.symbols = base + kOffArena;
  o.sym_cap = kArenaBytes - 256;
  o.sym_used = reinterpret_cast<unsigned long long *>(base + kOffUsed);
  o.pass_count = reinterpret_cast<uint32_t *>(base + kOffPcount);
  o.pass_off = reinterpret_cast<uint64_t *>(base + kOffPoff);
  launch_t1_encode(coeffs, reinterpret_cast<const CbDev *>(base + kOffCb), 1,
                   reinterpret_cast<const SbDev *>(base + kOffSb), o, (uint32_t)ncols, s);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    static_status_kernel<<<1, 1, 0, s>>>(base, status);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    fprintf(stderr, "bwc_b200_t1_encode_codeblock_static: %s\n", cudaGetErrorString(e));
    return 1;
  }
  return 0;
}
