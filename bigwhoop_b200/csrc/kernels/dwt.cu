// Multi-level separable CDF 9/7 and LeGall 5/3 lifting transforms, forward and inverse
// (dwt.c:354-466 9/7 lifting, :478-558 5/3 lifting, :286-342 boundary extension, :645-789
// de-/interleave, :1216-2246 level/axis drivers).
//
// Fields whose every transformed axis uses the 9/7 kernel take the fused paths below.  A field
// with a 5/3 axis, or a tile whose level regions start at odd coordinates, is transformed axis by
// axis in place (dwt_axis_kernel): each block holds whole lines in shared memory with an
// 8-sample reflected extension on both sides and lifts them over the extended range exactly as
// the reference lifts its extended line buffers, for either kernel and either start parity.
//
// Each level's spatial axes are transformed by one fused pass, reading one field-sized buffer
// and writing the other: the z-streaming kernel (dwt_stream_fwd_kernel) for large forward 3D
// levels, else dwt_level_kernel (a 3D tile with halos in shared memory, lifted along x, y and
// z, interior stored de-interleaved, or in natural order for the inverse); the time axis of 4D
// fields, when transformed, gets an in-place pass of its own (dwt_cols_kernel) in the
// reference's axis order.  Arithmetic is the reference's: float-literal lifting constants in
// the codec's type, a + c * (b0 + b1) with separately rounded products and sums, and
// whole-point symmetric extension of every line (repeated for lines shorter than the filter),
// which the tiles reproduce by loading reflected samples into their halos and lifting them
// like the reference lifts its extended lines.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "device_common.cuh"

namespace bwcb {
namespace {

// lifting constants: float literals widened to bwc_float (dwt.h:88-93)
constexpr bwc_float kAlpha = (bwc_float)-1.586134342059924f;
constexpr bwc_float kBeta = (bwc_float)-0.052980118572961f;
constexpr bwc_float kGamma = (bwc_float)0.882911075530934f;
constexpr bwc_float kDelta = (bwc_float)0.360523644801462f;
constexpr bwc_float kKappaH = (bwc_float)1.230174104914001f;
constexpr bwc_float kKappaL = (bwc_float)0.812893066115961f;

__device__ __forceinline__ int mirror(int i, int n) {
  // whole-point symmetric reflection into [0, n), repeated as often as needed
  while (i < 0 || i > n - 1) i = (i < 0) ? -i : 2 * (n - 1) - i;
  return i;
}

// one forward lifting update of sample i of a line held at w[j * stride], j in [0, n)
template <int kStep>
__device__ __forceinline__ void fwd_step(bwc_float *w, int n, int stride, int i) {
  const bwc_float a = w[mirror(i - 1, n) * stride];
  const bwc_float b = w[mirror(i + 1, n) * stride];
  bwc_float v = w[i * stride];
  if (kStep == 0) v = dev::fadd(v, dev::fmul(kAlpha, dev::fadd(a, b)));
  if (kStep == 1) v = dev::fadd(v, dev::fmul(kBeta, dev::fadd(a, b)));
  if (kStep == 2) v = dev::fmul(kKappaH, dev::fadd(v, dev::fmul(kGamma, dev::fadd(a, b))));
  if (kStep == 3) v = dev::fmul(kKappaL, dev::fadd(v, dev::fmul(kDelta, dev::fadd(a, b))));
  w[i * stride] = v;
}

// one inverse lifting update (dwt.c:416-466)
template <int kStep>
__device__ __forceinline__ void inv_step(bwc_float *w, int n, int stride, int i) {
  const bwc_float a = w[mirror(i - 1, n) * stride];
  const bwc_float b = w[mirror(i + 1, n) * stride];
  bwc_float v = w[i * stride];
  if (kStep == 0) v = dev::fsub(dev::fmul(kKappaH, v), dev::fmul(kDelta, dev::fadd(a, b)));
  if (kStep == 1) v = dev::fsub(dev::fmul(kKappaL, v), dev::fmul(kGamma, dev::fadd(a, b)));
  if (kStep == 2) v = dev::fsub(v, dev::fmul(kBeta, dev::fadd(a, b)));
  if (kStep == 3) v = dev::fsub(v, dev::fmul(kAlpha, dev::fadd(a, b)));
  w[i * stride] = v;
}

// ---- one axis in place: the time axis of 4D fields --------------------------------------------
// block (tx, ty): tile of TX consecutive x positions, whole line of length n along the axis
// with element stride `astride`; other coordinates: x-tile index, b (count eb, stride sb),
// c (stride sc).
template <bool kForward>
__global__ void __launch_bounds__(256) dwt_cols_kernel(bwc_float *__restrict__ work, int n, int TX,
                                                       uint32_t ex, uint64_t astride,
                                                       uint32_t eb, uint64_t sb, uint64_t sc,
                                                       uint32_t ntx) {
  extern __shared__ unsigned char smem_raw[];
  bwc_float *sm = reinterpret_cast<bwc_float *>(smem_raw);   // [n][TX]
  const uint32_t tile = blockIdx.x % ntx;
  const uint64_t bc = blockIdx.x / ntx;
  const uint64_t b = bc % eb, c = bc / eb;
  const uint32_t x0 = tile * TX;
  const int tw = (int)((ex - x0) < (uint32_t)TX ? (ex - x0) : (uint32_t)TX);
  bwc_float *base = work + x0 + b * sb + c * sc;
  const int half = (n + 1) >> 1;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int q = tid; q < n * TX; q += nth) {
    const int i = q / TX, x = q - i * TX;
    if (x < tw) {
      int j = i;
      if (!kForward) j = (i < half) ? 2 * i : 2 * (i - half) + 1;
      sm[j * TX + x] = base[(uint64_t)i * astride + x];
    }
  }
  __syncthreads();
  const int per_odd = n >> 1, per_even = (n + 1) >> 1;
#define COL_STEP(FN, K, PAR)                                                           \
  {                                                                                    \
    const int cnt = (PAR) ? per_odd : per_even;                                        \
    for (int q = tid; q < cnt * TX; q += nth) {                                        \
      const int k = q / TX, x = q - k * TX;                                            \
      if (x < tw) FN<K>(sm + x, n, TX, 2 * k + (PAR));                          \
    }                                                                                  \
    __syncthreads();                                                                   \
  }
  if (kForward) {
    COL_STEP(fwd_step, 0, 1)
    COL_STEP(fwd_step, 1, 0)
    COL_STEP(fwd_step, 2, 1)
    COL_STEP(fwd_step, 3, 0)
  } else {
    COL_STEP(inv_step, 0, 0)
    COL_STEP(inv_step, 1, 1)
    COL_STEP(inv_step, 2, 0)
    COL_STEP(inv_step, 3, 1)
  }
#undef COL_STEP
  for (int q = tid; q < n * TX; q += nth) {
    const int i = q / TX, x = q - i * TX;
    if (x < tw) {
      int j = i;
      if (kForward) j = (i < half) ? 2 * i : 2 * (i - half) + 1;
      base[(uint64_t)i * astride + x] = sm[j * TX + x];
    }
  }
}

constexpr size_t kSmemBudget = 96 * 1024;

template <bool kForward>
void cols_pass(bwc_float *work, const FieldDims &d, const uint64_t *e, int axis, cudaStream_t s) {
  const int n = (int)e[axis];
  const uint64_t stride[4] = {1, d.width, d.width * d.height, d.width * d.height * d.depth};
  int TX = 32;
  while (TX > 1 && (size_t)n * TX * sizeof(bwc_float) > kSmemBudget) TX >>= 1;
  const uint32_t ex = (uint32_t)e[0];
  const uint32_t ntx = (ex + TX - 1) / TX;
  // the two remaining axes
  int ob[2], k = 0;
  for (int a = 1; a < 4; ++a)
    if (a != axis) ob[k++] = a;
  const uint32_t eb = (uint32_t)e[ob[0]];
  const uint64_t nblocks = (uint64_t)ntx * e[ob[0]] * e[ob[1]];
  const size_t smem = (size_t)n * TX * sizeof(bwc_float);
  auto kern = dwt_cols_kernel<kForward>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget);
  kern<<<(unsigned)nblocks, 256, smem, s>>>(work, n, TX, ex, stride[axis], eb, stride[ob[0]],
                                            stride[ob[1]], ntx);
}

// ---- fused x/y/z pass of one level ---------------------------------------------------------
// One CTA transforms a tile of the level's region along every transformed spatial axis at once:
// it loads the tile plus a 4-sample halo on each side of every transformed axis (whole-point
// symmetric reflection at the region's edges, exactly the reference's line extension), lifts
// along x, then y, then z in shared memory (forward; z, y, x for the inverse), and stores the
// tile's interior -- de-interleaved (lows first) for the forward transform, in natural order for
// the inverse.  Four lifting steps of radius one make every interior sample exact with a
// 4-sample halo.  Tiles read `src` and write `dst`, two different buffers, so no tile can see
// another tile's output.
//
// Tile: 32 x 16 x 16 samples with halos (interior 24 x 8 x 8 along transformed axes, the whole
// 32 / 16 / 16 along untransformed ones).  Global loads and stores go a row per warp, so they
// are contiguous; the lifting runs on whole lines held in registers, one line per thread, so
// each axis costs one shared-memory read and write per sample.
constexpr int kLX = 32, kLY = 16, kLZ = 16, kH = 4;
constexpr int kFusedThreads = 256;

struct LevelGeom {
  uint32_t ex, ey, ez;       // region extents
  uint32_t tx, ty, tz;       // interior tile extents (24 / 8 / 8 or 32 / 16 / 16)
  uint32_t hx, hy, hz;       // halos (4 or 0)
  uint32_t ntx, nty, ntz;    // tiles per axis
  uint64_t sy, sz, st;       // buffer strides
};

__device__ __forceinline__ int reflect(int i, int n) {
  while (i < 0 || i > n - 1) i = (i < 0) ? -i : 2 * (n - 1) - i;
  return i;
}

// forward / inverse lifting step kStep at s[0] with neighbours s[-d], s[+d] (dwt.c:354-466)
template <bool kFwd, int kStep>
__device__ __forceinline__ void lift_at(bwc_float *s, int d) {
  const bwc_float ab = dev::fadd(s[-d], s[d]);
  bwc_float v = s[0];
  if (kFwd) {
    if (kStep == 0) v = dev::fadd(v, dev::fmul(kAlpha, ab));
    if (kStep == 1) v = dev::fadd(v, dev::fmul(kBeta, ab));
    if (kStep == 2) v = dev::fmul(kKappaH, dev::fadd(v, dev::fmul(kGamma, ab)));
    if (kStep == 3) v = dev::fmul(kKappaL, dev::fadd(v, dev::fmul(kDelta, ab)));
  } else {
    if (kStep == 0) v = dev::fsub(dev::fmul(kKappaH, v), dev::fmul(kDelta, ab));
    if (kStep == 1) v = dev::fsub(dev::fmul(kKappaL, v), dev::fmul(kGamma, ab));
    if (kStep == 2) v = dev::fsub(v, dev::fmul(kBeta, ab));
    if (kStep == 3) v = dev::fsub(v, dev::fmul(kAlpha, ab));
  }
  s[0] = v;
}

// The four lifting steps of one line held in registers (positions 0 and L-1 have only one
// neighbour inside the tile and are never updated; the halo makes them irrelevant).
template <bool kFwd, int L>
__device__ __forceinline__ void lift_line(bwc_float (&v)[L]) {
  // forward: odd, even, odd, even; inverse: even, odd, even, odd
  constexpr int p0 = kFwd ? 1 : 0, p1 = 1 - p0;
#pragma unroll
  for (int i = 1; i < L - 1; ++i)
    if ((i & 1) == p0) {
      const bwc_float ab = dev::fadd(v[i - 1], v[i + 1]);
      v[i] = kFwd ? dev::fadd(v[i], dev::fmul(kAlpha, ab))
                  : dev::fsub(dev::fmul(kKappaH, v[i]), dev::fmul(kDelta, ab));
    }
#pragma unroll
  for (int i = 1; i < L - 1; ++i)
    if ((i & 1) == p1) {
      const bwc_float ab = dev::fadd(v[i - 1], v[i + 1]);
      v[i] = kFwd ? dev::fadd(v[i], dev::fmul(kBeta, ab))
                  : dev::fsub(dev::fmul(kKappaL, v[i]), dev::fmul(kGamma, ab));
    }
#pragma unroll
  for (int i = 1; i < L - 1; ++i)
    if ((i & 1) == p0) {
      const bwc_float ab = dev::fadd(v[i - 1], v[i + 1]);
      v[i] = kFwd ? dev::fmul(kKappaH, dev::fadd(v[i], dev::fmul(kGamma, ab)))
                  : dev::fsub(v[i], dev::fmul(kBeta, ab));
    }
#pragma unroll
  for (int i = 1; i < L - 1; ++i)
    if ((i & 1) == p1) {
      const bwc_float ab = dev::fadd(v[i - 1], v[i + 1]);
      v[i] = kFwd ? dev::fmul(kKappaL, dev::fadd(v[i], dev::fmul(kDelta, ab)))
                  : dev::fsub(v[i], dev::fmul(kAlpha, ab));
    }
}

// shared-memory tile: rows of kLX samples padded to kPX, so that a warp whose lanes each walk
// their own row touches 32 different bank pairs
constexpr int kPX = kLX + 1;

__device__ __forceinline__ int tix(int x, int y, int z) { return (z * kLY + y) * kPX + x; }

// the x-rows with y in [y_lo, y_hi) and z in [z_lo, z_hi), one row per thread
template <bool kFwd>
__device__ __forceinline__ void lift_x(bwc_float *sm, int y_lo, int y_hi, int z_lo, int z_hi) {
  static_assert(kLY * kLZ == kFusedThreads, "one x-row per thread");
  const int y = threadIdx.x % kLY, z = threadIdx.x / kLY;
  if (y >= y_lo && y < y_hi && z >= z_lo && z < z_hi) {
    bwc_float v[kLX];
    bwc_float *row = sm + threadIdx.x * kPX;
#pragma unroll
    for (int i = 0; i < kLX; ++i) v[i] = row[i];
    lift_line<kFwd, kLX>(v);
#pragma unroll
    for (int i = 0; i < kLX; ++i) row[i] = v[i];
  }
  __syncthreads();
}

// the y-columns (kAxis 1) or z-columns (kAxis 2) with x in [x_lo, x_hi) and the remaining
// coordinate (z for y-columns, y for z-columns) in [o_lo, o_hi); lanes walk consecutive x
template <bool kFwd, int kAxis>
__device__ __forceinline__ void lift_yz(bwc_float *sm, int x_lo, int x_hi, int o_lo, int o_hi) {
  constexpr int L = (kAxis == 1) ? kLY : kLZ;
  constexpr int d = (kAxis == 1) ? kPX : kPX * kLY;
  const int x = threadIdx.x & 31;
  if (x >= x_lo && x < x_hi) {
    for (int o = o_lo + (threadIdx.x >> 5); o < o_hi; o += kFusedThreads / 32) {
      bwc_float *col = sm + ((kAxis == 1) ? tix(x, 0, o) : tix(x, o, 0));
      bwc_float v[L];
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = col[i * d];
      lift_line<kFwd, L>(v);
#pragma unroll
      for (int i = 0; i < L; ++i) col[i * d] = v[i];
    }
  }
  __syncthreads();
}

// asynchronous global -> shared copy of one sample (no register staging, many in flight)
__device__ __forceinline__ void copy_async(bwc_float *dst_smem, const bwc_float *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  if (sizeof(bwc_float) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}

// position of natural index g of an axis of extent e in the de-interleaved layout
__device__ __forceinline__ uint32_t mallat(uint32_t g, uint32_t e, bool on) {
  return on ? ((g & 1) ? ((e + 1) >> 1) + (g >> 1) : (g >> 1)) : g;
}

template <bool kFwd>
__global__ void __launch_bounds__(kFusedThreads)
    dwt_level_kernel(const bwc_float *__restrict__ src, bwc_float *__restrict__ dst,
                     LevelGeom g) {
  extern __shared__ unsigned char smem_raw[];
  bwc_float *sm = reinterpret_cast<bwc_float *>(smem_raw);
  uint32_t b = blockIdx.x;
  const uint32_t bx = b % g.ntx;
  b /= g.ntx;
  const uint32_t by = b % g.nty;
  b /= g.nty;
  const uint32_t bz = b % g.ntz;
  const uint32_t t = b / g.ntz;
  const int x0 = (int)(bx * g.tx) - (int)g.hx;
  const int y0 = (int)(by * g.ty) - (int)g.hy;
  const int z0 = (int)(bz * g.tz) - (int)g.hz;
  const bool onx = g.hx != 0, ony = g.hy != 0, onz = g.hz != 0;
  const bwc_float *sbase = src + (uint64_t)t * g.st;
  bwc_float *dbase = dst + (uint64_t)t * g.st;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Row offsets, one per thread (kLY * kLZ == kFusedThreads): the source row of each tile row
  // (reflected on transformed axes, clamped on untransformed ones -- clamped values are never
  // stored) and the destination row of each interior row (~0 where it lies outside the region).
  __shared__ uint64_t row_src[kLY * kLZ], row_dst[kLY * kLZ];
  {
    const int ly = threadIdx.x % kLY, lz = threadIdx.x / kLY;
    int gy = y0 + ly, gz = z0 + lz;
    const bool inside = gy >= 0 && gz >= 0 && gy < (int)g.ey && gz < (int)g.ez &&
                        ly >= (int)g.hy && ly < (int)(g.hy + g.ty) && lz >= (int)g.hz &&
                        lz < (int)(g.hz + g.tz);
    row_dst[threadIdx.x] =
        inside ? (uint64_t)(kFwd ? mallat((uint32_t)gy, g.ey, ony) : (uint32_t)gy) * g.sy +
                     (uint64_t)(kFwd ? mallat((uint32_t)gz, g.ez, onz) : (uint32_t)gz) * g.sz
               : ~0ull;
    gy = ony ? reflect(gy, (int)g.ey) : min(gy, (int)g.ey - 1);
    gz = onz ? reflect(gz, (int)g.ez) : min(gz, (int)g.ez - 1);
    row_src[threadIdx.x] =
        (uint64_t)(kFwd ? (uint32_t)gy : mallat((uint32_t)gy, g.ey, ony)) * g.sy +
        (uint64_t)(kFwd ? (uint32_t)gz : mallat((uint32_t)gz, g.ez, onz)) * g.sz;
  }
  __syncthreads();
  // load: one x-row per warp iteration, all rows in flight at once
  {
    int gx = x0 + lane;
    gx = onx ? reflect(gx, (int)g.ex) : min(gx, (int)g.ex - 1);
    const bwc_float *lsrc = sbase + (kFwd ? (uint32_t)gx : mallat((uint32_t)gx, g.ex, onx));
    bwc_float *ldst = sm + lane;
#pragma unroll 8
    for (int r = warp; r < kLY * kLZ; r += kFusedThreads / 32)
      copy_async(ldst + r * kPX, lsrc + row_src[r]);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  __syncthreads();
  // Lift every line along each transformed axis whose samples can reach the stored interior:
  // forward x on all rows, y on interior x, z on interior x and y; inverse z on all columns, y
  // on interior z, x on interior y and z.
  const int ix0 = (int)g.hx, ix1 = (int)(g.hx + g.tx);
  if (kFwd) {
    if (onx) lift_x<true>(sm, 0, kLY, 0, kLZ);
    if (ony) lift_yz<true, 1>(sm, ix0, ix1, 0, kLZ);
    if (onz) lift_yz<true, 2>(sm, ix0, ix1, (int)g.hy, (int)(g.hy + g.ty));
  } else {
    if (onz) lift_yz<false, 2>(sm, 0, kLX, 0, kLY);
    if (ony) lift_yz<false, 1>(sm, 0, kLX, (int)g.hz, (int)(g.hz + g.tz));
    if (onx) lift_x<false>(sm, (int)g.hy, (int)(g.hy + g.ty), (int)g.hz, (int)(g.hz + g.tz));
  }
  // store the interior
  {
    const int lx = ix0 + lane;
    const uint32_t gx = (uint32_t)(x0 + lx);
    if (lane < (int)g.tx && gx < g.ex) {
      bwc_float *sdst = dbase + (kFwd ? mallat(gx, g.ex, onx) : gx);
      for (int r = warp; r < kLY * kLZ; r += kFusedThreads / 32) {
        const uint64_t o = row_dst[r];
        if (o != ~0ull) sdst[o] = sm[r * kPX + lx];
      }
    }
  }
}

// ---- z-streaming forward pass of one level -------------------------------------------------
// For levels that transform x, y and z.  The level is cut into 64 x 64 tiles of (x, y) -- a
// 56 x 56 interior plus a 4-sample reflected halo on each side -- times pairs of z-planes; each
// CTA (one per SM) takes an equal share of those (tile, plane pair) units and streams through
// them, a contiguous run of planes of one tile at a time (with 4 reflected or neighbouring planes
// before the run and 3 to 4 after it).  Per plane:
//   x: the tile's rows come from global memory straight into registers, one plane ahead of use;
//      a warp holds a row as 32 (even, odd) pairs and lifts it with neighbours fetched by
//      shuffle; the row goes to a shared-memory plane split by row parity (rows of kZP samples);
//   y: the same warp-wide lifting on columns, each lane holding an (even row, odd row) pair of
//      two adjacent columns, read and written back as 16-byte words;
//   z: every lane keeps, for each of its points, a window of four planes in registers.  When an
//      even plane j has arrived, the lifting steps advance at planes j-1, j-2, j-3 and j-4 (the
//      only steps whose neighbours are complete), after which planes j-4 (low) and j-3 (high)
//      are final and stored de-interleaved.
// The three passes are software-pipelined over a ring of four plane slots: step s lifts plane s
// along x, plane s-1 along y and (s-2 even) planes s-3, s-2 along z, then one barrier.
// The arithmetic of every sample is the line lifting of dwt_level_kernel -- the same operands in
// the same order, rounded the same way -- only the z steps are scheduled as the planes arrive.
// Shuffles at the warp's ends read the lane's own value: those samples are halo, and a 4-sample
// halo keeps the interior exact, as for the tile kernel.  Samples a run reads before its first
// plane (a ring slot or window left by the previous run, or zeros) reach no stored sample.
constexpr int kZT = 64, kZH = 4, kZI = kZT - 2 * kZH;  // tile extent, halo, interior (x and y)
constexpr int kZThreads = 512;                           // 16 warps
constexpr int kZP = kZT + 2;                             // row pitch of a parity plane
constexpr int kZRing = 4;                                // tile planes held in shared memory
constexpr int kZPar = (kZT / 2) * kZP, kZSlot = 2 * kZPar;
constexpr size_t kZSmem = (size_t)kZRing * kZSlot * sizeof(bwc_float);

struct StreamGeom {
  uint32_t ex, ey, ez;        // region extents
  uint32_t lx, ly, lz;        // low-band sizes, (e + 1) / 2
  uint32_t ntx, nty, npairs;  // tiles along x and y, plane pairs along z
  uint32_t vec;               // rows start on pair boundaries: pair loads allowed
  uint32_t sy, sz;            // buffer strides within a time slice (< 2^31 samples)
  uint64_t st;                // time-slice stride
  uint64_t units;             // ntx * nty * time slices * npairs
};

template <typename T>
struct PairOf;
template <>
struct PairOf<double> {
  using type = double2;
};
template <>
struct PairOf<float> {
  using type = float2;
};
using pair_t = PairOf<bwc_float>::type;

template <int N>
__device__ __forceinline__ void shfl_down1(bwc_float (&d)[N], const bwc_float (&s)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) d[i] = __shfl_down_sync(0xffffffffu, s[i], 1);
}
template <int N>
__device__ __forceinline__ void shfl_up1(bwc_float (&d)[N], const bwc_float (&s)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) d[i] = __shfl_up_sync(0xffffffffu, s[i], 1);
}

// Forward lifting of N independent 64-sample lines, each held by the warp as (even, odd) pairs
// e[i], o[i] in lane order: odd samples take alpha from their even neighbours, evens beta from
// their odd neighbours, then gamma (scaled by kappa_H) and delta (scaled by kappa_L).
template <int N>
__device__ __forceinline__ void lift_pairs_fwd(bwc_float (&e)[N], bwc_float (&o)[N]) {
  bwc_float nb[N];
  shfl_down1(nb, e);
#pragma unroll
  for (int i = 0; i < N; ++i) o[i] = dev::fadd(o[i], dev::fmul(kAlpha, dev::fadd(e[i], nb[i])));
  shfl_up1(nb, o);
#pragma unroll
  for (int i = 0; i < N; ++i) e[i] = dev::fadd(e[i], dev::fmul(kBeta, dev::fadd(nb[i], o[i])));
  shfl_down1(nb, e);
#pragma unroll
  for (int i = 0; i < N; ++i)
    o[i] = dev::fmul(kKappaH, dev::fadd(o[i], dev::fmul(kGamma, dev::fadd(e[i], nb[i]))));
  shfl_up1(nb, o);
#pragma unroll
  for (int i = 0; i < N; ++i)
    e[i] = dev::fmul(kKappaL, dev::fadd(e[i], dev::fmul(kDelta, dev::fadd(nb[i], o[i]))));
}

__global__ void __launch_bounds__(kZThreads, 1)
    dwt_stream_fwd_kernel(const bwc_float *__restrict__ src, bwc_float *__restrict__ dst,
                          StreamGeom g) {
  extern __shared__ unsigned char smem_raw[];
  // ring[slot][row parity][row / 2][kZP]
  bwc_float *ring = reinterpret_cast<bwc_float *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kZRing * kZSlot; i += kZThreads) ring[i] = (bwc_float)0;
  // this thread's place in a slot: x and z passes (row warp + 16 k, lane's x pair), y pass
  // (column pairs warp and warp + 16, lane's row pair)
  const int xoff = (warp & 1) * kZPar + (warp >> 1) * kZP + 2 * lane;
  const int yoff = lane * kZP + 2 * warp;
  const int klo = (warp < kZH) ? 1 : 0, khi = (warp >= 16 - kZH) ? 3 : 4;   // interior rows

  // z window per point (row k, x parity i): w5 = plane j-5 after step 3, w4 = j-4 after step 2,
  // w3 = j-3 after step 1, w2 = j-2 as lifted along x and y
  bwc_float w5[4][2], w4[4][2], w3[4][2], w2[4][2];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int i = 0; i < 2; ++i) w5[k][i] = w4[k][i] = w3[k][i] = w2[k][i] = (bwc_float)0;
  __syncthreads();   // ring zeroed

  const uint64_t ubeg = (uint64_t)blockIdx.x * g.units / gridDim.x;
  const uint64_t uend = (uint64_t)(blockIdx.x + 1) * g.units / gridDim.x;
  for (uint64_t u = ubeg; u < uend;) {
    // the run: tile `tile`, plane pairs [p0, p1)
    const uint64_t tile = u / g.npairs;
    const uint32_t p0 = (uint32_t)(u % g.npairs);
    const uint64_t left = uend - u;
    const uint32_t p1 = (left < (uint64_t)(g.npairs - p0)) ? p0 + (uint32_t)left : g.npairs;
    u += p1 - p0;
    const uint32_t bx = (uint32_t)(tile % g.ntx);
    const uint32_t by = (uint32_t)((tile / g.ntx) % g.nty);
    const uint64_t t = tile / ((uint64_t)g.ntx * g.nty);
    const int x0 = (int)(bx * kZI) - kZH, y0 = (int)(by * kZI) - kZH;   // both even
    const int zc0 = 2 * (int)p0, zc1 = min(2 * (int)p1, (int)g.ez);
    const int jfirst = zc0 - kZH, jlast = (zc1 + 3) & ~1;   // first / last plane fed (even)
    const bwc_float *sbase = src + t * g.st;
    bwc_float *dbase = dst + t * g.st;

    // source offsets of this thread's rows, reflected; destination rows (~0u: not stored)
    const int xo = x0 + 2 * lane;
    const bool xin = x0 >= 0 && x0 + kZT <= (int)g.ex;
    const bool vec = xin && g.vec;
    const int xa = xin ? xo : reflect(xo, (int)g.ex);
    const int xb = xin ? xo + 1 : reflect(xo + 1, (int)g.ex);
    uint32_t lrow[4], srow[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int y = y0 + warp + 16 * k;
      lrow[k] = (uint32_t)reflect(y, (int)g.ey) * g.sy;
      const uint32_t yp = (y & 1) ? g.ly + (uint32_t)y / 2 : (uint32_t)y / 2;
      srow[k] = (k >= klo && k < khi && y < (int)g.ey) ? yp * g.sy : ~0u;
    }
    const uint32_t xe = (uint32_t)xo;
    const bool lane_in = lane >= kZH / 2 && lane < 32 - kZH / 2;
    const bool st_l = lane_in && xe < g.ex, st_h = lane_in && xe + 1 < g.ex;
    const uint32_t xl = xe / 2, xh = g.lx + xe / 2;

    auto load_plane = [&](int j, bwc_float (&e)[4], bwc_float (&o)[4]) {
      const bwc_float *p = sbase + (uint64_t)((uint32_t)reflect(j, (int)g.ez) * g.sz);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bwc_float *row = p + lrow[k];
        if (vec) {
          const pair_t v = __ldg(reinterpret_cast<const pair_t *>(row + xa));
          e[k] = v.x;
          o[k] = v.y;
        } else {
          e[k] = __ldg(row + xa);
          o[k] = __ldg(row + xb);
        }
      }
    };
    auto x_pass = [&](bwc_float (&e)[4], bwc_float (&o)[4], bwc_float *slot) {
      lift_pairs_fwd<4>(e, o);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        pair_t v;
        v.x = e[k];
        v.y = o[k];
        *reinterpret_cast<pair_t *>(slot + xoff + 8 * k * kZP) = v;   // row warp + 16 k
      }
    };
    auto y_pass = [&](bwc_float *slot) {
      bwc_float *ev = slot + yoff;
      bwc_float *od = ev + kZPar;
      bwc_float e[4], o[4];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const pair_t a = *reinterpret_cast<const pair_t *>(ev + 32 * q);
        const pair_t c = *reinterpret_cast<const pair_t *>(od + 32 * q);
        e[2 * q] = a.x;
        e[2 * q + 1] = a.y;
        o[2 * q] = c.x;
        o[2 * q + 1] = c.y;
      }
      lift_pairs_fwd<4>(e, o);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        pair_t a, c;
        a.x = e[2 * q];
        a.y = e[2 * q + 1];
        c.x = o[2 * q];
        c.y = o[2 * q + 1];
        *reinterpret_cast<pair_t *>(ev + 32 * q) = a;
        *reinterpret_cast<pair_t *>(od + 32 * q) = c;
      }
    };
    // z pass at even plane j: planes j-1 (odd) and j (even) enter the window
    auto z_pass = [&](int j, const bwc_float *slot_o, const bwc_float *slot_e) {
      const int ze = j - 4, zo = j - 3;
      const bool st_e = ze >= zc0 && ze < zc1, st_o = zo >= zc0 && zo < zc1;
      const uint32_t de = (uint32_t)(ze >> 1) * g.sz;
      const uint32_t dz = (g.lz + (uint32_t)(zo >> 1)) * g.sz;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k < klo || k >= khi) continue;
        const pair_t n0 = *reinterpret_cast<const pair_t *>(slot_e + xoff + 8 * k * kZP);
        const pair_t n1 = *reinterpret_cast<const pair_t *>(slot_o + xoff + 8 * k * kZP);
        bwc_float out_e[2], out_o[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const bwc_float v0 = i ? n0.y : n0.x;
          bwc_float v1 = i ? n1.y : n1.x;
          v1 = dev::fadd(v1, dev::fmul(kAlpha, dev::fadd(w2[k][i], v0)));
          w2[k][i] = dev::fadd(w2[k][i], dev::fmul(kBeta, dev::fadd(w3[k][i], v1)));
          w3[k][i] = dev::fmul(
              kKappaH, dev::fadd(w3[k][i], dev::fmul(kGamma, dev::fadd(w4[k][i], w2[k][i]))));
          w4[k][i] = dev::fmul(
              kKappaL, dev::fadd(w4[k][i], dev::fmul(kDelta, dev::fadd(w5[k][i], w3[k][i]))));
          out_e[i] = w4[k][i];
          out_o[i] = w3[k][i];
          w5[k][i] = w3[k][i];
          w4[k][i] = w2[k][i];
          w3[k][i] = v1;
          w2[k][i] = v0;
        }
        if (srow[k] != ~0u) {
          if (st_e) {
            if (st_l) dbase[de + srow[k] + xl] = out_e[0];
            if (st_h) dbase[de + srow[k] + xh] = out_e[1];
          }
          if (st_o) {
            if (st_l) dbase[dz + srow[k] + xl] = out_o[0];
            if (st_h) dbase[dz + srow[k] + xh] = out_o[1];
          }
        }
      }
    };

    // one register plane: plane s + 1 is requested as soon as the x pass has consumed plane s
    bwc_float pe_[4], po_[4];
    load_plane(jfirst, pe_, po_);
    for (int s = jfirst; s <= jlast + 2; ++s) {
      if (s <= jlast) {
        x_pass(pe_, po_, ring + (s & 3) * kZSlot);
        if (s < jlast) load_plane(s + 1, pe_, po_);
      }
      if (s - 1 >= jfirst && s - 1 <= jlast) y_pass(ring + ((s - 1) & 3) * kZSlot);
      if (s - 2 >= jfirst && ((s - 2) & 1) == 0)
        z_pass(s - 2, ring + ((s - 3) & 3) * kZSlot, ring + ((s - 2) & 3) * kZSlot);
      __syncthreads();
    }
  }
}

// ---- z-streaming forward levels staged by TMA tensor copies ---------------------------------
//
// dwt_tma_fwd_kernel: 40 x 40 (x, y) tiles -- a 32 x 32 interior with a 4-sample reflected halo
// -- streamed along z in batches of 8 planes, one CTA of 16 warps per SM.  A batch arrives in
// shared memory by TMA tensor copies completing on the batch slot's mbarrier: the interior
// columns as 128-byte-wide boxes with the 128-byte swizzle (16-byte chunk c of tile row y at
// chunk c ^ (y & 7), so row-wise and column-wise accesses are both conflict-free), and the two
// 4-column halos as narrow boxes.  A batch inside the region's z extent is one 3D box per column
// group (4 copies in FP64); a batch that reaches past either z end is loaded plane by plane with
// the reflected plane index.  Rows and columns outside the region (filled with zeros by TMA) are
// read from their reflected places: the thread that lifts a row reads the reflected source row,
// and the x-halo samples past the region's ends from the reflected place in that row.  Two batch
// slots: while a batch is lifted, the next one is in flight.  Per batch, one thread per tile row
// lifts the whole row along x in registers, one thread per interior column lifts the column
// along y, and each thread advances the z window of two interior points through the batch's
// planes and stores the finished coefficients in their de-interleaved places.  No shuffles:
// every line sits in one thread's registers.  The arithmetic of every sample is the tile
// kernel's line lifting (x, then y, then z), so the coefficients are bit-identical.  TMA wants
// 16-byte aligned rows (even widths in FP64, multiples of 4 in FP32); other fields take the
// kernels above.
constexpr int kBT = 40, kBH = 4, kBI = kBT - 2 * kBH;   // tile extent (x and y), halo, interior
constexpr int kBPl = 8;                                  // planes per batch
constexpr int kBThreads = 512;                           // 16 warps
constexpr int kES = (int)sizeof(bwc_float);
constexpr int kIB = 128 / kES;                   // samples per interior box row (128 bytes)
constexpr int kNIB = kBI / kIB;                  // interior boxes (FP64 2, FP32 1)
constexpr int kPerChunk = 16 / kES;              // samples per 16-byte chunk
constexpr int kHW = kBH;                         // halo box width
constexpr uint32_t kIBPlane = kBT * 128;                     // bytes of an interior box plane
constexpr uint32_t kIBBytes = kBPl * kIBPlane;               // ... of an interior box
constexpr uint32_t kHPlane = kBT * kHW * kES;                // ... of a halo box plane
constexpr uint32_t kHBytes = kBPl * kHPlane;                 // ... of a halo box
constexpr uint32_t kHaloL = kNIB * kIBBytes, kHaloR = kHaloL + kHBytes;
constexpr uint32_t kSlotBytes = kHaloR + kHBytes;            // one batch slot
constexpr size_t kBSmem = 1024 + 2 * (size_t)kSlotBytes + 128;   // + alignment, barriers
constexpr uint32_t kBSpin = 1u << 22;   // mbarrier polls before a batch is given up
static_assert(kSlotBytes % 1024 == 0 && kIBBytes % 1024 == 0 && kIBPlane % 1024 == 0,
              "swizzled boxes start on 1024-byte boundaries");
static_assert(kHaloL % 128 == 0 && kHPlane % 128 == 0, "halo boxes start on 128-byte boundaries");
static_assert(kBThreads >= kBPl * kBT, "one thread per row of a batch");
static_assert(kBThreads / 32 >= kBPl && kBI == 32, "one warp per plane in the y pass");
static_assert(kBPl * (kNIB + 2) <= 32, "one warp issues a batch's per-plane copies");

struct BulkGeom {
  uint32_t ex, ey, ez;      // region extents
  uint32_t lx, ly, lz;      // low-band sizes, (e + 1) / 2
  uint32_t ntx, nty, nbat;  // tiles along x and y, 8-plane output batches along z
  uint32_t sy, sz;          // buffer strides within a time slice (< 2^31 samples)
  uint64_t st;              // time-slice stride
  uint32_t units;           // ntx * nty * time slices * nbat (< 2^31)
};

// tensor maps over the level region (x, y, z, t): interior and halo boxes, 8 planes deep and
// one plane deep
struct TmaMaps {
  CUtensorMap in8, halo8, in1, halo1;
};

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};
using v16_t = Vec16<bwc_float>::type;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// bounded wait for the phase of the given parity; false when it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kBSpin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// TMA tensor copy of the box at (x, y, z, t) into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                         int t, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(t), "r"(smem_u32(bar))
      : "memory");
}

// byte offset in a slot of tile sample i (0..39) of row y of plane p
__device__ __forceinline__ uint32_t tma_off(int p, int y, int i) {
  const uint32_t r = (uint32_t)(p * kBT + y);
  if (i < kBH) return kHaloL + (r * kHW + (uint32_t)i) * kES;
  if (i >= kBH + kBI) return kHaloR + (r * kHW + (uint32_t)(i - kBH - kBI)) * kES;
  const int xi = i - kBH, bx = xi / kIB, e = xi % kIB;
  const uint32_t c = (uint32_t)(e / kPerChunk) ^ (uint32_t)(y & 7);
  return (uint32_t)bx * kIBBytes + r * 128 + c * 16 + (uint32_t)(e % kPerChunk) * kES;
}

// A CTA's units form runs (consecutive output batches of one tile column); a run's fed planes
// are zc0 - 5 (odd) .. (zc1 + 3) & ~1 (even): four context planes on either side of its output
// planes [zc0, zc1), and (odd, even) plane pairs inside every batch of 8.
struct BulkRun {
  uint32_t u, n;   // first unit, units
  int nb;          // batches fed
};
__device__ __forceinline__ BulkRun bulk_run(const BulkGeom &g, uint32_t u, uint32_t uend) {
  BulkRun r;
  r.u = u;
  if (u >= uend) {
    r.n = 0;
    r.nb = 0;
    return r;
  }
  const uint32_t b0 = u % g.nbat;
  r.n = min(uend - u, g.nbat - b0);
  const int zc0 = kBPl * (int)b0, zc1 = min(kBPl * (int)(b0 + r.n), (int)g.ez);
  r.nb = ((((zc1 + 3) & ~1) - (zc0 - 5) + 1) + kBPl - 1) / kBPl;
  return r;
}

// batch k of a run, as every thread of the CTA reads it from shared memory
struct BulkBatch {
  uint32_t bx, by, t;
  int zc0, zc1;   // output planes of the run
  int jb, np;     // first fed plane, planes (even, <= 8); np = 0: no batch
  int whole;      // planes jb .. jb + np - 1 lie inside the region: one 3D box per column group
};
__device__ __forceinline__ BulkBatch bulk_batch(const BulkGeom &g, const BulkRun &r, int k) {
  BulkBatch b;
  b.np = 0;
  if (r.n == 0) return b;
  const uint32_t tile = r.u / g.nbat, b0 = r.u % g.nbat;
  b.bx = tile % g.ntx;
  const uint32_t rest = tile / g.ntx;
  b.by = rest % g.nty;
  b.t = rest / g.nty;
  b.zc0 = kBPl * (int)b0;
  b.zc1 = min(kBPl * (int)(b0 + r.n), (int)g.ez);
  b.jb = b.zc0 - 5 + kBPl * k;
  b.np = min(kBPl, ((b.zc1 + 3) & ~1) + 1 - b.jb);
  b.whole = b.jb >= 0 && b.jb + b.np <= (int)g.ez;
  return b;
}
// bytes one batch brings into its slot (boxes count whole, zero-filled parts included)
__device__ __forceinline__ uint32_t bulk_bytes(const BulkBatch &b) {
  return b.whole ? kSlotBytes : (uint32_t)b.np * (kNIB * kIBPlane + 2 * kHPlane);
}

__global__ void __launch_bounds__(kBThreads, 1)
    dwt_tma_fwd_kernel(bwc_float *__restrict__ dst, BulkGeom g, const __grid_constant__ TmaMaps maps,
                       uint32_t *fault) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // swizzled boxes want 1024-byte aligned destinations
  unsigned char *sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * (size_t)kSlotBytes);
  BulkBatch *desc = reinterpret_cast<BulkBatch *>(bar + 2);   // the batch in each slot
  volatile int &s_abort = *reinterpret_cast<int *>(desc + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const uint32_t ubeg = (uint32_t)((uint64_t)blockIdx.x * g.units / gridDim.x);
  const uint32_t uend = (uint32_t)((uint64_t)(blockIdx.x + 1) * g.units / gridDim.x);
  // the posting thread (the first of the last warp, idle in the x and y passes) walks the
  // batch sequence one batch ahead of the issue: (arun, ak) is the next batch to post
  BulkRun arun = bulk_run(g, ubeg, uend);
  int ak = 0;
  auto advance = [&]() {
    if (++ak >= arun.nb) {
      arun = bulk_run(g, arun.u + arun.n, uend);
      ak = 0;
    }
  };
  // the posting thread writes a slot's batch and arrives on the slot's barrier with the batch's
  // bytes (the one arrival of each phase) before any copy of it is issued
  auto post = [&](uint32_t q) {
    const BulkBatch b = bulk_batch(g, arun, ak);
    desc[q & 1] = b;
    if (b.np) {
      advance();
      mbar_arrive_tx(&bar[q & 1], bulk_bytes(b));
    }
  };
  if (tid == kBThreads - 32) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&maps.in8))
                 : "memory");
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&maps.halo8))
                 : "memory");
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    post(0);
    post(1);
  }
  __syncthreads();

  // warp 0 issues the copies of the batch described in slot q & 1
  auto issue = [&](uint32_t q) {
    const BulkBatch b = desc[q & 1];
    if (warp != 0 || b.np == 0) return;
    const uint32_t base = smem_u32(sm) + (q & 1) * kSlotBytes;
    const int xb = (int)(b.bx * kBI), yb = (int)(b.by * kBI) - kBH;
    // copy `lane`: box kind k (0 .. kNIB-1 interior, kNIB left halo, kNIB+1 right halo), plane p
    const int k = lane % (kNIB + 2), p = lane / (kNIB + 2);
    const int x = (k < kNIB) ? xb + k * kIB : (k == kNIB ? xb - kBH : xb + kBI);
    const uint32_t kb = (k < kNIB) ? (uint32_t)k * kIBBytes : (k == kNIB ? kHaloL : kHaloR);
    if (b.whole) {
      if (p == 0)
        tma_load(base + kb, (k < kNIB) ? &maps.in8 : &maps.halo8, x, yb, b.jb, (int)b.t, &bar[q & 1]);
    } else if (p < b.np) {
      const uint32_t pb = (k < kNIB) ? kIBPlane : kHPlane;
      tma_load(base + kb + (uint32_t)p * pb, (k < kNIB) ? &maps.in1 : &maps.halo1, x, yb,
               reflect(b.jb + p, (int)g.ez), (int)b.t, &bar[q & 1]);
    }
  };
  issue(0);
  issue(1);

  // y- and z-pass column of this lane (column 4 + lane): sample of row y at
  // cb + (c16 ^ 16 (y & 7)) + 128 y of its plane
  const uint32_t cb = (uint32_t)(lane / kIB) * kIBBytes + (uint32_t)(lane % kPerChunk) * kES;
  const uint32_t c16 = (uint32_t)((lane % kIB) / kPerChunk) * 16;

  // z windows of this thread's two interior points (column 4 + lane, rows 4 + warp and
  // 20 + warp): w5 = plane j-5 after step 3, w4 = j-4 after step 2, w3 = j-3 after step 1,
  // w2 = j-2 as lifted along x and y
  bwc_float w5[2], w4[2], w3[2], w2[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) w5[i] = w4[i] = w3[i] = w2[i] = (bwc_float)0;

  uint32_t q = 0;
  for (;; ++q) {
    const BulkBatch b = desc[q & 1];
    if (b.np == 0) break;
    unsigned char *slot = sm + (q & 1) * kSlotBytes;
    const bool arrived = mbar_wait(&bar[q & 1], (q >> 1) & 1);
    if (!arrived) s_abort = 1;
    const int x0 = (int)(b.bx * kBI) - kBH, y0 = (int)(b.by * kBI) - kBH;
    const bool yedge = y0 < 0 || y0 + kBT > (int)g.ey;

    // rows just outside the region (4 on either side) first take their reflected source row;
    // rows further out feed no stored sample and keep the zeros TMA wrote
    const int p = tid / kBT, y = tid % kBT;
    const bool xrow = tid < kBT * b.np && arrived;
    if (yedge) {
      const int yy = y0 + y;
      if (xrow && ((yy < 0 && yy >= -kBH) || (yy >= (int)g.ey && yy < (int)g.ey + kBH))) {
        const int ys = reflect(yy, (int)g.ey) - y0;
        const uint32_t rd = (uint32_t)(p * kBT + y), rs = (uint32_t)(p * kBT + ys);
#pragma unroll
        for (int i = 0; i < kHW; i += kPerChunk) {
          *reinterpret_cast<v16_t *>(slot + kHaloL + (rd * kHW + i) * kES) =
              *reinterpret_cast<const v16_t *>(slot + kHaloL + (rs * kHW + i) * kES);
          *reinterpret_cast<v16_t *>(slot + kHaloR + (rd * kHW + i) * kES) =
              *reinterpret_cast<const v16_t *>(slot + kHaloR + (rs * kHW + i) * kES);
        }
#pragma unroll
        for (int c = 0; c < kBI / kPerChunk; ++c) {
          const uint32_t bo = (uint32_t)(c / (kIB / kPerChunk)) * kIBBytes;
          const uint32_t cc = (uint32_t)(c % (kIB / kPerChunk));
          *reinterpret_cast<v16_t *>(slot + bo + rd * 128 + ((cc ^ (uint32_t)(y & 7)) * 16)) =
              *reinterpret_cast<const v16_t *>(slot + bo + rs * 128 + ((cc ^ (uint32_t)(ys & 7)) * 16));
        }
      }
      __syncthreads();
    }

    // x pass: one row per thread; x-halo samples just past the region's ends come from their
    // reflected place in the row (further out: zeros, feeding no stored sample)
    if (xrow) {
      bwc_float v[kBT];
      const uint32_t r = (uint32_t)(p * kBT + y);
#pragma unroll
      for (int i = 0; i < kHW; i += kPerChunk) {
        const v16_t a = *reinterpret_cast<const v16_t *>(slot + kHaloL + (r * kHW + i) * kES);
        const v16_t c = *reinterpret_cast<const v16_t *>(slot + kHaloR + (r * kHW + i) * kES);
#pragma unroll
        for (int e = 0; e < kPerChunk; ++e) {
          v[i + e] = reinterpret_cast<const bwc_float *>(&a)[e];
          v[kBH + kBI + i + e] = reinterpret_cast<const bwc_float *>(&c)[e];
        }
      }
#pragma unroll
      for (int c = 0; c < kBI / kPerChunk; ++c) {
        const uint32_t o = (uint32_t)(c / (kIB / kPerChunk)) * kIBBytes + r * 128 +
                           ((uint32_t)(c % (kIB / kPerChunk)) ^ (uint32_t)(y & 7)) * 16;
        const v16_t a = *reinterpret_cast<const v16_t *>(slot + o);
#pragma unroll
        for (int e = 0; e < kPerChunk; ++e)
          v[kBH + c * kPerChunk + e] = reinterpret_cast<const bwc_float *>(&a)[e];
      }
      if (x0 < 0) {   // x = -4 .. -1 reflect to 4 .. 1
#pragma unroll
        for (int i = 0; i < kBH; ++i) v[i] = v[2 * kBH - i];
      }
      if (x0 + kBT > (int)g.ex) {
#pragma unroll
        for (int i = kBH + 1; i < kBT; ++i) {
          const int xx = x0 + i;
          if (xx >= (int)g.ex && xx < (int)g.ex + kBH)
            v[i] = *reinterpret_cast<const bwc_float *>(
                slot + tma_off(p, y, reflect(xx, (int)g.ex) - x0));
        }
      }
      lift_line<true, kBT>(v);
#pragma unroll
      for (int c = 0; c < kBI / kPerChunk; ++c) {
        const uint32_t o = (uint32_t)(c / (kIB / kPerChunk)) * kIBBytes + r * 128 +
                           ((uint32_t)(c % (kIB / kPerChunk)) ^ (uint32_t)(y & 7)) * 16;
        v16_t a;
#pragma unroll
        for (int e = 0; e < kPerChunk; ++e)
          reinterpret_cast<bwc_float *>(&a)[e] = v[kBH + c * kPerChunk + e];
        *reinterpret_cast<v16_t *>(slot + o) = a;
      }
    }
    __syncthreads();
    if (s_abort) break;
    // the batch after next goes into this slot's record now (every thread holds this batch's
    // record and has passed this slot's wait); a warp the y pass leaves idle writes it
    if (tid == kBThreads - 32) post(q + 2);

    // y pass: one interior column per thread, one warp per plane
    if (warp < b.np) {
      unsigned char *col = slot + cb + (uint32_t)warp * kIBPlane;
      bwc_float v[kBT];
#pragma unroll
      for (int i = 0; i < kBT; ++i)
        v[i] = *reinterpret_cast<const bwc_float *>(col + (c16 ^ (16u * (i & 7))) + (uint32_t)i * 128);
      lift_line<true, kBT>(v);
#pragma unroll
      for (int i = kBH; i < kBH + kBI; ++i)
        *reinterpret_cast<bwc_float *>(col + (c16 ^ (16u * (i & 7))) + (uint32_t)i * 128) = v[i];
    }
    __syncthreads();

    // z pass: (odd, even) plane pairs (jb + p, jb + p + 1); at even plane j the finished planes
    // are j - 4 (low band) and j - 3 (high band)
    {
      bwc_float *dbase = dst + (uint64_t)b.t * g.st;
      const uint32_t gx = b.bx * kBI + (uint32_t)lane;
      const uint32_t mx = (gx & 1) ? g.lx + (gx >> 1) : (gx >> 1);
      uint32_t off[2];
      bool in[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const uint32_t gy = b.by * kBI + (uint32_t)(warp + 16 * i);
        const uint32_t my = (gy & 1) ? g.ly + (gy >> 1) : (gy >> 1);
        off[i] = mx + my * g.sy;
        in[i] = gx < g.ex && gy < g.ey;
      }
      // rows 4 + warp and 20 + warp share y & 7; all four plane pairs are lifted (past np, in a
      // run's last batch, they read earlier planes and change only the window, which the next
      // run's context planes refill before any of its stored samples)
      const unsigned char *pt =
          slot + cb + (c16 ^ (16u * ((kBH + warp) & 7))) + (uint32_t)(kBH + warp) * 128;
#pragma unroll
      for (int pp = 0; pp < kBPl; pp += 2) {
        const int j = b.jb + pp + 1;
        const int ze = j - 4, zo = j - 3;
        const bool st_e = ze >= b.zc0 && ze < b.zc1, st_o = zo >= b.zc0 && zo < b.zc1;
        const uint32_t de = (uint32_t)(ze >> 1) * g.sz;
        const uint32_t dz = (g.lz + (uint32_t)(zo >> 1)) * g.sz;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const bwc_float v1 =
              *reinterpret_cast<const bwc_float *>(pt + (uint32_t)pp * kIBPlane + 16u * 128u * i);
          const bwc_float v0 = *reinterpret_cast<const bwc_float *>(
              pt + (uint32_t)(pp + 1) * kIBPlane + 16u * 128u * i);
          const bwc_float a = dev::fadd(v1, dev::fmul(kAlpha, dev::fadd(w2[i], v0)));
          const bwc_float c = dev::fadd(w2[i], dev::fmul(kBeta, dev::fadd(w3[i], a)));
          const bwc_float o = dev::fmul(
              kKappaH, dev::fadd(w3[i], dev::fmul(kGamma, dev::fadd(w4[i], c))));
          const bwc_float e = dev::fmul(
              kKappaL, dev::fadd(w4[i], dev::fmul(kDelta, dev::fadd(w5[i], o))));
          if (in[i]) {
            if (st_e) dbase[de + off[i]] = e;
            if (st_o) dbase[dz + off[i]] = o;
          }
          w5[i] = o;
          w4[i] = c;
          w3[i] = a;
          w2[i] = v0;
        }
      }
    }
    __syncthreads();   // the slot is consumed
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    issue(q + 2);
  }
  if (s_abort) {
    if (tid == 0) atomicOr(fault, 1u);
    // the other slot's copies may still be in flight: wait for them (bounded) before leaving
    if (desc[(q + 1) & 1].np) mbar_wait(&bar[(q + 1) & 1], ((q + 1) >> 1) & 1);
  }
}

// ---- one axis in place, any kernel ---------------------------------------------------------
constexpr int kExt = 8;   // reflected samples on each side of a line (the liftings read at most 6)
// LeGall 5/3 lifting constants of the reference (dwt.c:478-558): halving and (sum + 2) / 4
constexpr bwc_float kTwo = (bwc_float)2, kFour = (bwc_float)4;

// Lines of length `len` along an axis of element stride `sa` (the region's extent on that axis),
// TX of them side by side along the companion axis (extent ec, stride sc); blockIdx enumerates
// x tiles, then the two remaining axes (extent e1 with stride s1, then stride s2).  Forward: load
// the line, extend, lift, store lows first (a line starting at an odd coordinate, `odd`, lifts
// one sample further into the extension and takes its lows from w[0], w[2], ... and highs from
// w[-1], w[1], ...).  Inverse: load interleaved, extend, lift, store in natural order.
template <bool kFwd>
__global__ void __launch_bounds__(256) dwt_axis_kernel(bwc_float *__restrict__ work, int len,
                                                       int odd, int kern, uint64_t sa, int TX,
                                                       uint32_t ec, uint64_t sc, uint32_t e1,
                                                       uint64_t s1, uint64_t s2, uint32_t ntx) {
  extern __shared__ unsigned char smem_raw[];
  bwc_float *sm = reinterpret_cast<bwc_float *>(smem_raw);
  const int rows = len + 2 * kExt + 2;   // line positions -kExt-1 .. len+kExt
  const uint32_t tile = blockIdx.x % ntx;
  const uint64_t rest = blockIdx.x / ntx;
  const uint64_t i1 = rest % e1, i2 = rest / e1;
  const uint32_t c0 = tile * (uint32_t)TX;
  const int tw = (int)((ec - c0) < (uint32_t)TX ? (ec - c0) : (uint32_t)TX);
  bwc_float *base = work + (uint64_t)c0 * sc + i1 * s1 + i2 * s2;
  const int tid = threadIdx.x, nth = blockDim.x;
  // B[q] of line x at sm[(q + kExt + 1) * TX + x]; the lifting's w = B + odd
  auto B = [&](int q, int x) -> bwc_float & { return sm[(q + kExt + 1) * TX + x]; };
  const int half = odd ? (len >> 1) : ((len + 1) >> 1);
  if (!kFwd && odd && (len & 1)) {
    // the inverse's fill leaves this sample unwritten (the line's last high lands past its end,
    // where the extension overwrites it); it is zero here
    for (int x = tid; x < TX; x += nth) B(len - 1, x) = (bwc_float)0;
  }
  for (int q = tid; q < len * TX; q += nth) {
    const int i = q / TX, x = q - i * TX;
    if (x >= tw) continue;
    const bwc_float v = base[(uint64_t)x * sc + (uint64_t)i * sa];
    if (kFwd) {
      B(i, x) = v;
    } else {
      // coefficient i of the stored line is interleaved back to position j
      const int j = (i < half) ? 2 * i : 2 * (i - half) + 1;
      B(j, x) = v;
    }
  }
  __syncthreads();
  // whole-point symmetric extension, reflected as often as needed (dwt.c:286-342)
  for (int q = tid; q < 2 * kExt * TX; q += nth) {
    const int k = q / TX, x = q - k * TX;
    if (x >= tw) continue;
    const int e = (k < kExt) ? -(k + 1) : len - 1 + (k - kExt + 1);
    int j = e;
    while (j < 0 || j > len - 1) j = (j < 0) ? -j : 2 * (len - 1) - j;
    B(e, x) = B(j, x);
  }
  __syncthreads();
  // one lifting step over w[i], i = i0, i0 + 2, ... < i1
  auto step = [&](int i0, int i1e, auto fn) {
    const int cnt = (i1e - i0 + 1) / 2;
    for (int q = tid; q < cnt * TX; q += nth) {
      const int k = q / TX, x = q - k * TX;
      if (x >= tw) continue;
      const int i = i0 + 2 * k + odd;
      B(i, x) = fn(B(i, x), B(i - 1, x), B(i + 1, x));
    }
    __syncthreads();
  };
  using dev::fadd;
  using dev::fdiv;
  using dev::fmul;
  using dev::fsub;
  if (kern == 1) {
    if (kFwd) {
      step(-1, len + 1, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(v, fdiv(fadd(a, b), kTwo)); });
      step(0, len, [](bwc_float v, bwc_float a, bwc_float b) { return fadd(v, fdiv(fadd(fadd(a, b), kTwo), kFour)); });
    } else {
      step(-2, len + 1, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(v, fdiv(fadd(fadd(a, b), kTwo), kFour)); });
      step(-1, len, [](bwc_float v, bwc_float a, bwc_float b) { return fadd(v, fdiv(fadd(a, b), kTwo)); });
    }
  } else {
    if (kFwd) {
      step(-3, len + 3, [](bwc_float v, bwc_float a, bwc_float b) { return fadd(v, fmul(kAlpha, fadd(a, b))); });
      step(-2, len + 2, [](bwc_float v, bwc_float a, bwc_float b) { return fadd(v, fmul(kBeta, fadd(a, b))); });
      step(-1, len + 1, [](bwc_float v, bwc_float a, bwc_float b) { return fmul(kKappaH, fadd(v, fmul(kGamma, fadd(a, b)))); });
      step(0, len, [](bwc_float v, bwc_float a, bwc_float b) { return fmul(kKappaL, fadd(v, fmul(kDelta, fadd(a, b)))); });
    } else {
      step(-4, len + 4, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(fmul(kKappaH, v), fmul(kDelta, fadd(a, b))); });
      step(-5, len + 3, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(fmul(kKappaL, v), fmul(kGamma, fadd(a, b))); });
      step(-4, len + 2, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(v, fmul(kBeta, fadd(a, b))); });
      step(-3, len + 1, [](bwc_float v, bwc_float a, bwc_float b) { return fsub(v, fmul(kAlpha, fadd(a, b))); });
    }
  }
  for (int q = tid; q < len * TX; q += nth) {
    const int i = q / TX, x = q - i * TX;
    if (x >= tw) continue;
    bwc_float v;
    if (kFwd) {
      // lows first: w[0], w[2], ...; then the highs
      v = (i < half) ? B(2 * i + odd, x) : B(2 * (i - half) + (odd ? -1 : 1) + odd, x);
    } else {
      v = B(i, x);
    }
    base[(uint64_t)x * sc + (uint64_t)i * sa] = v;
  }
}

// dst = src over the box [0, e0) x [0, e1) x [0, e2) x [0, e3) of the buffer
__global__ void __launch_bounds__(256) copy_region_kernel(const bwc_float *__restrict__ src,
                                                          bwc_float *__restrict__ dst,
                                                          uint32_t e0, uint32_t e1, uint32_t e2,
                                                          uint64_t rows, uint64_t sy, uint64_t sz,
                                                          uint64_t st) {
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const uint64_t y = r % e1, z = (r / e1) % e2, t = r / ((uint64_t)e1 * e2);
    const uint64_t base = y * sy + z * sz + t * st;
    for (uint32_t x = threadIdx.x; x < e0; x += blockDim.x) dst[base + x] = src[base + x];
  }
}

void copy_region(const bwc_float *src, bwc_float *dst, const FieldDims &d, const uint64_t *e,
                 cudaStream_t s) {
  const uint64_t rows = e[1] * e[2] * e[3];
  if (!rows || !e[0]) return;
  const unsigned grid = (unsigned)std::min<uint64_t>(rows, (uint64_t)dev::kNumSMs * 64);
  copy_region_kernel<<<grid, 256, 0, s>>>(src, dst, (uint32_t)e[0], (uint32_t)e[1],
                                          (uint32_t)e[2], rows, d.width, d.width * d.height,
                                          d.width * d.height * d.depth);
}

// Transform path selection (bwc_b200_set_transform_tuning): 0 = tile kernel only; 1 = the
// TMA streaming kernel wherever x, y and z are transformed, span at least 8 and rows start on
// 16-byte boundaries, else the register streaming kernel where x and y span at least
// 48 samples and the level gives every SM at least 8 plane pairs; 2 = as 1, with the register
// streaming kernel wherever x, y and z are transformed and span at least 8; 3 = the register
// streaming kernel wherever possible, never the TMA one.  `ctas` > 0 fixes the streaming
// kernels' grids, 0 = one CTA per SM.
int g_transform_mode = 1;
int g_transform_ctas = 0;

// set by a TMA streaming kernel whose batch did not arrive within its wait limit (never expected)
__device__ uint32_t g_dwt_fault;

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    n = dev::kNumSMs;
  return n;
}

uint32_t *fault_word() {
  static std::mutex m;
  static uint32_t *addr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(m);
  if (!addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dwt_fault) != cudaSuccess) return nullptr;
    addr[dev] = static_cast<uint32_t *>(p);
  }
  return addr[dev];
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  // initialised once, thread-safely (a function-local static)
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
  }();
  return fn;
}

// a 4D tensor map over the level region of `src` with boxes of bw x 40 x bz x 1
bool region_map(CUtensorMap *m, const bwc_float *src, const FieldDims &d, const uint64_t *e,
                uint32_t bw, uint32_t bz, bool swizzle) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[4] = {e[0], e[1], e[2], e[3]};
  const cuuint64_t strides[3] = {d.width * sizeof(bwc_float), d.width * d.height * sizeof(bwc_float),
                                 d.width * d.height * d.depth * sizeof(bwc_float)};
  const cuuint32_t box[4] = {bw, (cuuint32_t)kBT, bz, 1};
  const cuuint32_t unit[4] = {1, 1, 1, 1};
  const CUresult r =
      enc(m, sizeof(bwc_float) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
          4, const_cast<bwc_float *>(src), dims, strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
          swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
          // interior rows are 128 bytes; a halo row is 32 (FP64) or 16 bytes, and a larger L2
          // fetch for it read several times the field from DRAM (ncu at 256^3: 347 MB for 134)
          swizzle ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_NONE,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tma_pass(const bwc_float *src, bwc_float *dst, const FieldDims &d, const uint64_t *e,
              uint8_t on, cudaStream_t s) {
  if (g_transform_mode == 0 || g_transform_mode == 3 || (on & 7) != 7) return false;
  if (e[0] < 8 || e[1] < 8 || e[2] < 8) return false;
  if (d.width * d.height * d.depth >= (1ull << 31)) return false;   // 32-bit slice offsets
  const uint64_t es = sizeof(bwc_float);
  if ((reinterpret_cast<uintptr_t>(src) % 16) || (d.width * es) % 16) return false;
  uint32_t *fault = fault_word();
  if (!fault) return false;
  TmaMaps maps;
  if (!region_map(&maps.in8, src, d, e, kIB, kBPl, true) ||
      !region_map(&maps.halo8, src, d, e, kHW, kBPl, false) ||
      !region_map(&maps.in1, src, d, e, kIB, 1, true) ||
      !region_map(&maps.halo1, src, d, e, kHW, 1, false))
    return false;
  BulkGeom g;
  g.ex = (uint32_t)e[0];
  g.ey = (uint32_t)e[1];
  g.ez = (uint32_t)e[2];
  g.lx = (g.ex + 1) >> 1;
  g.ly = (g.ey + 1) >> 1;
  g.lz = (g.ez + 1) >> 1;
  g.ntx = (g.ex + kBI - 1) / kBI;
  g.nty = (g.ey + kBI - 1) / kBI;
  g.nbat = (g.ez + kBPl - 1) / kBPl;
  const uint64_t units = (uint64_t)g.ntx * g.nty * e[3] * g.nbat;
  if (units >= (1ull << 31)) return false;
  g.units = (uint32_t)units;
  g.sy = (uint32_t)d.width;
  g.sz = (uint32_t)(d.width * d.height);
  g.st = d.width * d.height * d.depth;
  static const int sms = sm_count();
  const uint64_t grid =
      std::min<uint64_t>(g.units, g_transform_ctas > 0 ? (uint64_t)g_transform_ctas : (uint64_t)sms);
  cudaFuncSetAttribute(dwt_tma_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kBSmem);
  dwt_tma_fwd_kernel<<<(unsigned)grid, kBThreads, kBSmem, s>>>(dst, g, maps, fault);
  return true;
}

bool stream_pass(const bwc_float *src, bwc_float *dst, const FieldDims &d, const uint64_t *e,
                 uint8_t on, cudaStream_t s) {
  if (tma_pass(src, dst, d, e, on, s)) return true;
  if (g_transform_mode == 0 || (on & 7) != 7) return false;
  if (e[0] < 8 || e[1] < 8 || e[2] < 8) return false;
  if (d.width * d.height * d.depth >= (1ull << 31)) return false;   // 32-bit slice offsets
  StreamGeom g;
  g.ex = (uint32_t)e[0];
  g.ey = (uint32_t)e[1];
  g.ez = (uint32_t)e[2];
  g.lx = (g.ex + 1) >> 1;
  g.ly = (g.ey + 1) >> 1;
  g.lz = (g.ez + 1) >> 1;
  g.ntx = (g.ex + kZI - 1) / kZI;
  g.nty = (g.ey + kZI - 1) / kZI;
  g.npairs = (g.ez + 1) / 2;
  g.units = (uint64_t)g.ntx * g.nty * e[3] * g.npairs;
  g.vec = (d.width % 2) == 0;
  g.sy = (uint32_t)d.width;
  g.sz = (uint32_t)(d.width * d.height);
  g.st = d.width * d.height * d.depth;
  static const int sms = sm_count();
  const uint64_t grid =
      std::min<uint64_t>(g.units, g_transform_ctas > 0 ? (uint64_t)g_transform_ctas : (uint64_t)sms);
  if (g_transform_mode == 1 && (e[0] < 48 || e[1] < 48 || g.units < 8 * grid)) return false;
  cudaFuncSetAttribute(dwt_stream_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kZSmem);
  dwt_stream_fwd_kernel<<<(unsigned)grid, kZThreads, kZSmem, s>>>(src, dst, g);
  return true;
}

template <bool kFwd>
void level_pass(const bwc_float *src, bwc_float *dst, const FieldDims &d, const uint64_t *e,
                uint8_t on, cudaStream_t s) {
  if (kFwd && stream_pass(src, dst, d, e, on, s)) return;
  LevelGeom g;
  g.ex = (uint32_t)e[0];
  g.ey = (uint32_t)e[1];
  g.ez = (uint32_t)e[2];
  g.hx = (on & 1) ? kH : 0;
  g.hy = (on & 2) ? kH : 0;
  g.hz = (on & 4) ? kH : 0;
  g.tx = kLX - 2 * g.hx;
  g.ty = kLY - 2 * g.hy;
  g.tz = kLZ - 2 * g.hz;
  g.ntx = (g.ex + g.tx - 1) / g.tx;
  g.nty = (g.ey + g.ty - 1) / g.ty;
  g.ntz = (g.ez + g.tz - 1) / g.tz;
  g.sy = d.width;
  g.sz = d.width * d.height;
  g.st = d.width * d.height * d.depth;
  const uint64_t blocks = (uint64_t)g.ntx * g.nty * g.ntz * e[3];
  const size_t smem = (size_t)kPX * kLY * kLZ * sizeof(bwc_float);
  auto k = dwt_level_kernel<kFwd>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<(unsigned)blocks, kFusedThreads, smem, s>>>(src, dst, g);
}

// one axis of a level's region in place with dwt_axis_kernel
template <bool kFwd>
void axis_pass(bwc_float *work, const FieldDims &d, const uint64_t *e, int a, int kern, int odd,
               cudaStream_t s) {
  const int len = (int)e[a];
  if (len <= 1) return;
  const uint64_t st[4] = {1, d.width, d.width * d.height, d.width * d.height * d.depth};
  const int c = (a == 0) ? 1 : 0;
  int o[2], k = 0;
  for (int b = 0; b < 4; ++b)
    if (b != a && b != c) o[k++] = b;
  const size_t line_bytes = (size_t)(len + 2 * kExt + 2) * sizeof(bwc_float);
  int TX = (int)std::min<size_t>(32, std::max<size_t>(1, (96 * 1024) / line_bytes));
  TX = (int)std::min<uint64_t>((uint64_t)TX, std::max<uint64_t>(1, e[c]));
  const uint32_t ntx = (uint32_t)((e[c] + TX - 1) / TX);
  const uint64_t blocks = (uint64_t)ntx * e[o[0]] * e[o[1]];
  if (!blocks) return;
  const size_t smem = line_bytes * TX;
  auto kf = dwt_axis_kernel<kFwd>;
  cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kf<<<(unsigned)blocks, 256, smem, s>>>(work, len, odd, kern, st[a], TX, (uint32_t)e[c], st[c],
                                         (uint32_t)e[o[0]], st[o[0]], st[o[1]], ntx);
}

bool uses_axis_path(const DwtPlan &plan) {
  for (int l = 0; l < plan.levels; ++l)
    for (int a = 0; a < 4; ++a)
      if ((plan.axis_on[l] >> a & 1) && (plan.kern[a] != 0 || (plan.odd[l] >> a & 1))) return true;
  return false;
}

}  // namespace

void dwt_setup() { fault_word(); }

void dwt_fault_download(uint32_t *host, cudaStream_t s) {
  uint32_t *f = fault_word();
  if (!f) {
    *host = 0;
    return;
  }
  cudaMemcpyAsync(host, f, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  cudaMemsetAsync(f, 0, sizeof(uint32_t), s);
}

// Forward: `temp` holds the normalised field on entry; the coefficients end in `work`.  Even
// levels go temp -> work and odd levels work -> temp, each level reading one buffer and writing
// the other.  The high bands a level leaves in temp (odd levels) are copied back to work before
// the next level overwrites the lows inside them, and after the last level.  The time axis of
// 4D fields is transformed by a separate in-place pass after the spatial axes of each level.
void launch_dwt_forward(bwc_float *work, bwc_float *temp, const FieldDims &dims,
                        const DwtPlan &plan, cudaStream_t s) {
  const uint64_t full[4] = {dims.width, dims.height, dims.depth, dims.dt};
  if (plan.levels == 0) {
    copy_region(temp, work, dims, full, s);
    return;
  }
  if (uses_axis_path(plan)) {
    // axis by axis in place (x, y, z, t per level), each with its own kernel
    copy_region(temp, work, dims, full, s);
    for (int l = 0; l < plan.levels; ++l)
      for (int a = 0; a < 4; ++a)
        if (plan.axis_on[l] >> a & 1)
          axis_pass<true>(work, dims, plan.ext[l], a, plan.kern[a], plan.odd[l] >> a & 1, s);
    return;
  }
  for (int l = 0; l < plan.levels; ++l) {
    const uint64_t *e = plan.ext[l];
    const bool even = (l % 2) == 0;
    const bwc_float *src = even ? temp : work;
    bwc_float *dst = even ? work : temp;
    if (even && l > 0) copy_region(temp, work, dims, plan.ext[l - 1], s);
    level_pass<true>(src, dst, dims, e, plan.axis_on[l] & 7, s);
    if (plan.axis_on[l] & 8) cols_pass<true>(dst, dims, e, 3, s);
  }
  if (plan.levels % 2 == 0) copy_region(temp, work, dims, plan.ext[plan.levels - 1], s);
}

// Inverse: `temp` holds the coefficients on entry (scratch afterwards); the field ends in
// `work`.  Level l reads temp when l is even and work when l is odd, so the odd levels' inputs
// (their high bands) are copied to work once at the start; every level's lows come from the
// level above, written into the buffer it reads.
void launch_dwt_inverse(bwc_float *work, bwc_float *temp, const FieldDims &dims,
                        const DwtPlan &plan, cudaStream_t s) {
  const uint64_t full[4] = {dims.width, dims.height, dims.depth, dims.dt};
  if (plan.levels == 0) {
    copy_region(temp, work, dims, full, s);
    return;
  }
  if (uses_axis_path(plan)) {
    // axis by axis in place (t, z, y, x per level, coarsest level first), then to `work`
    for (int l = plan.levels - 1; l >= 0; --l)
      for (int a = 3; a >= 0; --a)
        if (plan.axis_on[l] >> a & 1)
          axis_pass<false>(temp, dims, plan.ext[l], a, plan.kern[a], plan.odd[l] >> a & 1, s);
    copy_region(temp, work, dims, full, s);
    return;
  }
  if (plan.levels > 1) copy_region(temp, work, dims, plan.ext[1], s);
  for (int l = plan.levels - 1; l >= 0; --l) {
    const uint64_t *e = plan.ext[l];
    const bool even = (l % 2) == 0;
    bwc_float *src = even ? temp : work;
    bwc_float *dst = even ? work : temp;
    if (plan.axis_on[l] & 8) cols_pass<false>(src, dims, e, 3, s);
    level_pass<false>(src, dst, dims, e, plan.axis_on[l] & 7, s);
  }
}

}  // namespace bwcb

extern "C" void bwc_b200_set_transform_tuning(int mode, int ctas) {
  bwcb::g_transform_mode = (mode < 0 || mode > 3) ? 1 : mode;
  bwcb::g_transform_ctas = ctas > 0 ? ctas : 0;
}
