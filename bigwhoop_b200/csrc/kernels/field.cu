// Field conversion, range normalisation and the inverse (libbwc.c:622-812, :993-1176,
// :827-978): element-wise, HBM-bound streaming kernels.
//
//  fill_minmax : dtype -> bwc_float copy plus the global min/max (order-independent atomics on
//                order-preserving integer keys)
//  normalize   : f = (f - alpha) * beta, then exponent += Qm unless f is +-0 (exact x 2^Qm)
//  denormalize : exponent -= Qm unless +-0, f = f * beta' + alpha, converted to the output dtype
#include "device_common.cuh"

namespace bwcb {
namespace {

__device__ __forceinline__ uint64_t order_key(bwc_float f) {
  const uint64_t u = (uint64_t)dev::as_raw(f);
  const uint64_t sign = (uint64_t)kSignMask;
  return (u & sign) ? (~u & (sign | (sign - 1))) : (u | sign);
}

__device__ __forceinline__ bwc_float key_value(uint64_t k) {
  const uint64_t sign = (uint64_t)kSignMask;
  const uint64_t u = (k & sign) ? (k & ~sign) : (~k & (sign | (sign - 1)));
  return dev::as_float((bwc_raw)u);
}

template <typename Src>
__global__ void __launch_bounds__(256) fill_minmax_kernel(const Src *__restrict__ src,
                                                          uint64_t n, bwc_float *__restrict__ work,
                                                          uint64_t *keys) {
  uint64_t kmin = ~0ull, kmax = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bwc_float v = (bwc_float)src[i];
    work[i] = v;
    if (v == v) {
      const uint64_t k = order_key(v);
      kmin = min(kmin, k);
      kmax = max(kmax, k);
    }
  }
  for (int o = 16; o; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  }
  __shared__ uint64_t smin[8], smax[8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smin[w] = kmin;
    smax[w] = kmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 1; j < (int)(blockDim.x >> 5); ++j) {
      kmin = min(kmin, smin[j]);
      kmax = max(kmax, smax[j]);
    }
    if (kmin != ~0ull) atomicMin((unsigned long long *)&keys[0], (unsigned long long)kmin);
    if (kmax != 0) atomicMax((unsigned long long *)&keys[1], (unsigned long long)kmax);
  }
}

__global__ void __launch_bounds__(256) normalize_kernel(bwc_float *__restrict__ work, uint64_t n,
                                                        const uint64_t *keys, uint8_t Qm,
                                                        bwc_float *stats) {
  const bwc_float mn = key_value(keys[0]);
  const bwc_float mx = key_value(keys[1]);
  // alpha = (max + min) / 2.0f, beta = 2.0f / (max - min) in bwc_float arithmetic
  const bwc_float alpha = dev::fdiv(dev::fadd(mx, mn), (bwc_float)2.0f);
  const bwc_float beta = dev::fdiv((bwc_float)2.0f, dev::fsub(mx, mn));
  if (blockIdx.x == 0 && threadIdx.x == 0 && stats) {
    stats[0] = mn;
    stats[1] = mx;
    stats[2] = alpha;
    stats[3] = beta;
  }
  const bwc_raw shift = (bwc_raw)Qm << kPrecMantissa;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bwc_float f = dev::fmul(dev::fsub(work[i], alpha), beta);
    bwc_raw r = dev::as_raw(f);
    r += (((r & kExponentMask) == 0) && ((r & kMantissaMask) == 0)) ? 0 : shift;
    work[i] = dev::as_float(r);
  }
}

template <typename Dst>
__global__ void __launch_bounds__(256) denormalize_kernel(const bwc_float *__restrict__ work,
                                                          uint64_t n, bwc_float alpha,
                                                          bwc_float beta, uint8_t Qm,
                                                          Dst *__restrict__ dst) {
  const bwc_raw shift = (bwc_raw)Qm << kPrecMantissa;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bwc_raw r = dev::as_raw(work[i]);
    r -= (((r & kExponentMask) == 0) && ((r & kMantissaMask) == 0)) ? 0 : shift;
    const bwc_float f = dev::fadd(dev::fmul(dev::as_float(r), beta), alpha);
    dst[i] = (Dst)f;
  }
}

// element i of a box (x fastest) at field index base + x + sy*y + sz*z + st*t
__device__ __forceinline__ uint64_t box_index(const BoxMap &m, uint64_t i) {
  const uint64_t x = i % m.w;
  uint64_t r = i / m.w;
  const uint64_t y = r % m.h;
  r /= m.h;
  const uint64_t z = r % m.d, t = r / m.d;
  return m.base + x + m.sy * y + m.sz * z + m.st * t;
}

template <typename Src>
__global__ void __launch_bounds__(256) fill_box_minmax_kernel(const Src *__restrict__ src,
                                                              uint64_t n, BoxMap m,
                                                              bwc_float *__restrict__ work,
                                                              uint64_t *keys) {
  uint64_t kmin = ~0ull, kmax = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bwc_float v = (bwc_float)src[box_index(m, i)];
    work[i] = v;
    if (v == v) {
      const uint64_t k = order_key(v);
      kmin = min(kmin, k);
      kmax = max(kmax, k);
    }
  }
  for (int o = 16; o; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  }
  __shared__ uint64_t smin[8], smax[8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    smin[w] = kmin;
    smax[w] = kmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int j = 1; j < (int)(blockDim.x >> 5); ++j) {
      kmin = min(kmin, smin[j]);
      kmax = max(kmax, smax[j]);
    }
    if (kmin != ~0ull) atomicMin((unsigned long long *)&keys[0], (unsigned long long)kmin);
    if (kmax != 0) atomicMax((unsigned long long *)&keys[1], (unsigned long long)kmax);
  }
}

template <typename Dst>
__global__ void __launch_bounds__(256) denormalize_box_kernel(const bwc_float *__restrict__ work,
                                                              uint64_t n, bwc_float alpha,
                                                              bwc_float beta, uint8_t Qm,
                                                              Dst *__restrict__ dst, BoxMap m) {
  const bwc_raw shift = (bwc_raw)Qm << kPrecMantissa;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bwc_raw r = dev::as_raw(work[i]);
    r -= (((r & kExponentMask) == 0) && ((r & kMantissaMask) == 0)) ? 0 : shift;
    const bwc_float f = dev::fadd(dev::fmul(dev::as_float(r), beta), alpha);
    dst[box_index(m, i)] = (Dst)f;
  }
}

unsigned grid_for(uint64_t n) {
  const uint64_t per = 256ull * 8;
  uint64_t g = (n + per - 1) / per;
  const uint64_t cap = (uint64_t)dev::kNumSMs * 16;
  if (g > cap) g = cap;
  return (unsigned)(g ? g : 1);
}

}  // namespace

void launch_fill_minmax(const void *src, bool src_double, uint64_t n, bwc_float *work,
                        uint64_t *keys, cudaStream_t s) {
  if (src_double)
    fill_minmax_kernel<double><<<grid_for(n), 256, 0, s>>>((const double *)src, n, work, keys);
  else
    fill_minmax_kernel<float><<<grid_for(n), 256, 0, s>>>((const float *)src, n, work, keys);
}

void launch_fill_minmax_box(const void *src, bool src_double, uint64_t n, const BoxMap &m,
                            bwc_float *work, uint64_t *keys, cudaStream_t s) {
  if (src_double)
    fill_box_minmax_kernel<double><<<grid_for(n), 256, 0, s>>>((const double *)src, n, m, work, keys);
  else
    fill_box_minmax_kernel<float><<<grid_for(n), 256, 0, s>>>((const float *)src, n, m, work, keys);
}

void launch_denormalize_box(const bwc_float *work, uint64_t n, bwc_float pmin, bwc_float pmax,
                            uint8_t Qm, void *dst, bool dst_double, const BoxMap &m,
                            cudaStream_t s) {
  const bwc_float alpha = (bwc_float)((pmax + pmin) / (bwc_float)2.0f);
  const bwc_float beta = (bwc_float)((pmax - pmin) / (bwc_float)2.0f);
  if (dst_double)
    denormalize_box_kernel<double><<<grid_for(n), 256, 0, s>>>(work, n, alpha, beta, Qm, (double *)dst, m);
  else
    denormalize_box_kernel<float><<<grid_for(n), 256, 0, s>>>(work, n, alpha, beta, Qm, (float *)dst, m);
}

void launch_normalize(bwc_float *work, uint64_t n, const uint64_t *keys, uint8_t Qm,
                      bwc_float *stats, cudaStream_t s) {
  normalize_kernel<<<grid_for(n), 256, 0, s>>>(work, n, keys, Qm, stats);
}

void launch_denormalize(const bwc_float *work, uint64_t n, bwc_float pmin, bwc_float pmax,
                        uint8_t Qm, void *dst, bool dst_double, cudaStream_t s) {
  // alpha = (max + min) / 2.0f, beta = (max - min) / 2.0f, on the host in bwc_float
  const bwc_float alpha = (bwc_float)((pmax + pmin) / (bwc_float)2.0f);
  const bwc_float beta = (bwc_float)((pmax - pmin) / (bwc_float)2.0f);
  if (dst_double)
    denormalize_kernel<double><<<grid_for(n), 256, 0, s>>>(work, n, alpha, beta, Qm, (double *)dst);
  else
    denormalize_kernel<float><<<grid_for(n), 256, 0, s>>>(work, n, alpha, beta, Qm, (float *)dst);
}

}  // namespace bwcb
