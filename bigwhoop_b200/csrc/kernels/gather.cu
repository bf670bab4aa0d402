// Byte gather: assembles a codestream from host-built header bytes and slices of the device
// tier-1 buffer (compression), or the per-codeblock coded bytes from the slices scattered over
// packets of an input codestream (decompression).  One warp per piece, 16-byte vector copies
// where source and destination are co-aligned.
#include "device_common.cuh"

namespace bwcb {
namespace {

__global__ void __launch_bounds__(256) gather_kernel(uint8_t *__restrict__ dst,
                                                     const uint8_t *__restrict__ blob,
                                                     const uint8_t *__restrict__ devsrc,
                                                     const GatherPiece *__restrict__ pieces,
                                                     uint64_t npieces) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t w = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < npieces;
       w += nw) {
    const GatherPiece p = pieces[w];
    const uint8_t *src = (p.from_blob ? blob : devsrc) + p.src;
    uint8_t *d = dst + p.dst;
    uint64_t n = p.size, i = 0;
    if ((((uintptr_t)src ^ (uintptr_t)d) & 15) == 0) {
      const uint64_t head = (16 - ((uintptr_t)d & 15)) & 15;
      for (uint64_t k = lane; k < head && k < n; k += 32) d[k] = src[k];
      i = head < n ? head : n;
      const uint64_t nvec = (n - i) >> 4;
      const uint4 *s4 = reinterpret_cast<const uint4 *>(src + i);
      uint4 *d4 = reinterpret_cast<uint4 *>(d + i);
      for (uint64_t k = lane; k < nvec; k += 32) d4[k] = s4[k];
      i += nvec << 4;
    }
    for (uint64_t k = i + lane; k < n; k += 32) d[k] = src[k];
  }
}

}  // namespace

void launch_gather(uint8_t *dst, const uint8_t *blob, const uint8_t *dev, const GatherPiece *pieces,
                   uint64_t npieces, cudaStream_t s) {
  if (!npieces) return;
  uint64_t blocks = (npieces + 7) / 8;
  if (blocks > (uint64_t)dev::kNumSMs * 8) blocks = (uint64_t)dev::kNumSMs * 8;
  gather_kernel<<<(unsigned)blocks, 256, 0, s>>>(dst, blob, dev, pieces, npieces);
}

}  // namespace bwcb
