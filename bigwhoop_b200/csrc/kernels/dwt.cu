// Multi-level separable CDF 9/7 lifting transform, forward and inverse
// (dwt.c:354-466 lifting, :286-342 boundary extension, :645-789 de-/interleave,
// :1216-2246 level/axis drivers).
//
// Lines are staged in shared memory and lifted in place with four data-parallel steps.  The
// reference extends each line by whole-point symmetric reflection (repeated for lines shorter
// than the filter) and lifts the extension too; since reflection preserves index parity and
// each lifting step updates mirrored samples with mirrored operands, reading neighbours through
// the reflected index gives bit-identical results for every sample inside the line, which is
// what is done here.  Arithmetic is the reference's: float-literal lifting constants in the
// codec's type, a + c * (b0 + b1) with separately rounded products and sums.
//
//   rows kernel  (x axis): one CTA per group of rows, lines contiguous in HBM;
//   cols kernel  (y/z/t axes): one CTA per tile of consecutive x columns and its whole line,
//                 loaded as coalesced x-rows and lifted column-wise.
// After lifting, even samples (low-pass) are stored first, odd samples (high-pass) after them.
#include <algorithm>
#include <cstdio>

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

// ---- x axis: rows --------------------------------------------------------------------------
// block handles `rows` consecutive lines (index r -> (y, z, t) within the region)
template <bool kForward>
__global__ void __launch_bounds__(256) dwt_rows_kernel(bwc_float *__restrict__ work, int n,
                                                       int rows_per_block, uint64_t nlines,
                                                       uint32_t ey, uint32_t ez,
                                                       uint64_t row_stride, uint64_t slab_stride,
                                                       uint64_t vol_stride) {
  extern __shared__ unsigned char smem_raw[];
  bwc_float *sm = reinterpret_cast<bwc_float *>(smem_raw);
  const uint64_t first = (uint64_t)blockIdx.x * rows_per_block;
  const uint64_t left = nlines - first;
  const int nrows = (int)(left < (uint64_t)rows_per_block ? left : (uint64_t)rows_per_block);
  const int half = (n + 1) >> 1;
  // load (forward: natural order; inverse: interleave lows/highs)
  for (int r = 0; r < nrows; ++r) {
    const uint64_t line = first + r;
    const uint64_t y = line % ey, z = (line / ey) % ez, t = line / ((uint64_t)ey * ez);
    const bwc_float *src = work + y * row_stride + z * slab_stride + t * vol_stride;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int j = i;
      if (!kForward) j = (i < half) ? 2 * i : 2 * (i - half) + 1;
      sm[r * n + j] = src[i];
    }
  }
  __syncthreads();
  // each lifting step updates the samples of one parity of every row in parallel
  const int tid = threadIdx.x, nth = blockDim.x;
  const int per_row_odd = n >> 1, per_row_even = (n + 1) >> 1;
#define ROW_STEP(FN, K, PAR)                                                           \
  {                                                                                    \
    const int cnt = (PAR) ? per_row_odd : per_row_even;                                \
    for (int q = tid; q < nrows * cnt; q += nth) {                                     \
      const int r = q / cnt, i = 2 * (q - r * cnt) + (PAR);                            \
      FN<K>(sm + r * n, n, 1, i);                                               \
    }                                                                                  \
    __syncthreads();                                                                   \
  }
  if (kForward) {
    ROW_STEP(fwd_step, 0, 1)
    ROW_STEP(fwd_step, 1, 0)
    ROW_STEP(fwd_step, 2, 1)
    ROW_STEP(fwd_step, 3, 0)
  } else {
    ROW_STEP(inv_step, 0, 0)
    ROW_STEP(inv_step, 1, 1)
    ROW_STEP(inv_step, 2, 0)
    ROW_STEP(inv_step, 3, 1)
  }
#undef ROW_STEP
  for (int r = 0; r < nrows; ++r) {
    const uint64_t line = first + r;
    const uint64_t y = line % ey, z = (line / ey) % ez, t = line / ((uint64_t)ey * ez);
    bwc_float *dst = work + y * row_stride + z * slab_stride + t * vol_stride;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int j = i;
      if (kForward) j = (i < half) ? 2 * i : 2 * (i - half) + 1;
      dst[i] = sm[r * n + j];
    }
  }
}

// ---- y/z/t axes: columns ---------------------------------------------------------------------
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
void rows_pass(bwc_float *work, const FieldDims &d, const uint64_t *e, cudaStream_t s) {
  const int n = (int)e[0];
  const uint64_t nlines = e[1] * e[2] * e[3];
  int rows = (int)std::max<size_t>(1, std::min<size_t>(kSmemBudget / (n * sizeof(bwc_float)),
                                                       (size_t)std::max(1, 4096 / n)));
  const size_t smem = (size_t)rows * n * sizeof(bwc_float);
  const uint64_t blocks = (nlines + rows - 1) / rows;
  auto k = dwt_rows_kernel<kForward>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget);
  k<<<(unsigned)blocks, 256, smem, s>>>(work, n, rows, nlines, (uint32_t)e[1], (uint32_t)e[2],
                                        d.width, d.width * d.height,
                                        d.width * d.height * d.depth);
}

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

}  // namespace

void launch_dwt_forward(bwc_float *work, const FieldDims &dims, const DwtPlan &plan,
                        cudaStream_t s) {
  for (int l = 0; l < plan.levels; ++l) {
    const uint64_t *e = plan.ext[l];
    if (plan.axis_on[l] & 1) rows_pass<true>(work, dims, e, s);
    for (int a = 1; a < 4; ++a)
      if (plan.axis_on[l] & (1 << a)) cols_pass<true>(work, dims, e, a, s);
  }
}

void launch_dwt_inverse(bwc_float *work, const FieldDims &dims, const DwtPlan &plan,
                        cudaStream_t s) {
  for (int l = plan.levels - 1; l >= 0; --l) {
    const uint64_t *e = plan.ext[l];
    for (int a = 3; a >= 1; --a)
      if (plan.axis_on[l] & (1 << a)) cols_pass<false>(work, dims, e, a, s);
    if (plan.axis_on[l] & 1) rows_pass<false>(work, dims, e, s);
  }
}

}  // namespace bwcb
