// Statevector reductions: norm^2 (FP64 accumulation) and scaling.
//
// Replaces src/cpp/cuda/cuda_kernels.cu of narix10yc/cast_simulator
// (normSqPass1/2 at :124-167, scaleKernel at :171-196, C wrappers at :244-254).
// Same two-pass structure - per-block FP64 partial sums over 128-bit loads into
// a device scratch array, then one block folds the partials - but sized for
// B200: 4 blocks of 256 threads per SM, 4 independent 128-bit loads in flight
// per thread per iteration.  Both run on the legacy default stream, as the
// reference's do (cuda_kernels.cu:236-238), so they order after earlier work on
// blocking streams.
#include "../../include/ffi_cuda.h"
#include "internal.hpp"

#include <mutex>

namespace cb2 {

namespace {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double part[kRedThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  v = threadIdx.x < kRedThreads / 32 ? part[threadIdx.x] : 0.0;
  if (threadIdx.x < 32) v = warp_sum(v);
  return v;
}

__device__ __forceinline__ double sq4(float4 v) {
  return (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
}
__device__ __forceinline__ double sq4(double2 v) { return v.x * v.x + v.y * v.y; }

template <typename T> struct V16;
template <> struct V16<float> { using type = float4; static constexpr int N = 4; };
template <> struct V16<double> { using type = double2; static constexpr int N = 2; };

// Pass 1: partial[blockIdx.x] = sum of squares of this block's share.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_norm_pass1(const T *__restrict__ x, uint64_t n,
                                                           double *__restrict__ partial) {
  using V = typename V16<T>::type;
  constexpr int N = V16<T>::N;
  const V *xv = reinterpret_cast<const V *>(x);
  const uint64_t nv = n / N;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (; i + 3 * stride < nv; i += 4 * stride) {
    const V v0 = xv[i], v1 = xv[i + stride], v2 = xv[i + 2 * stride], v3 = xv[i + 3 * stride];
    a0 += sq4(v0);
    a1 += sq4(v1);
    a2 += sq4(v2);
    a3 += sq4(v3);
  }
  for (; i < nv; i += stride) a0 += sq4(xv[i]);
  double acc = (a0 + a1) + (a2 + a3);
  // scalar tail (n not a multiple of the vector width)
  if (blockIdx.x == 0 && threadIdx.x < n - nv * N) {
    const double t = (double)x[nv * N + threadIdx.x];
    acc += t * t;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Pass 2: out[0] = sum of the partials (one block).
__global__ void __launch_bounds__(kRedThreads) k_norm_pass2(const double *__restrict__ partial,
                                                            int n, double *__restrict__ out) {
  double acc = 0;
  for (int i = threadIdx.x; i < n; i += kRedThreads) acc += partial[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[0] = acc;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_scale(T *__restrict__ x, uint64_t n, T s) {
  using V = typename V16<T>::type;
  constexpr int N = V16<T>::N;
  V *xv = reinterpret_cast<V *>(x);
  const uint64_t nv = n / N;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  for (uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; i < nv; i += stride) {
    V v = xv[i];
    if constexpr (N == 4) {
      v.x *= s; v.y *= s; v.z *= s; v.w *= s;
    } else {
      v.x *= s; v.y *= s;
    }
    xv[i] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * N) x[nv * N + threadIdx.x] *= s;
}

// Scratch: partial sums + the final value, allocated once per process and
// grown on demand (the reference keeps the same kind of process-wide scratch,
// cuda_kernels.cu:203-230).  The mutex serialises users of the scratch.
std::mutex g_scratch_mu;
double *g_scratch = nullptr;
int g_scratch_len = 0;

bool ensure_scratch(int len, std::string &err) {
  if (g_scratch && g_scratch_len >= len) return true;
  if (g_scratch) cudaFree(g_scratch);
  g_scratch = nullptr;
  g_scratch_len = 0;
  if (!cuda_ok(cudaMalloc(&g_scratch, sizeof(double) * len), "cudaMalloc (norm scratch)", err))
    return false;
  g_scratch_len = len;
  return true;
}

unsigned red_grid(uint64_t nv) {
  const uint64_t want = (nv + kRedThreads - 1) / kRedThreads;
  const uint64_t cap = 4ull * sm_count();
  return (unsigned)std::max<uint64_t>(1, std::min(want, cap));
}

template <typename T>
bool norm_sq_impl(const void *x, uint64_t n, double *out, cudaStream_t s, std::string &err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned grid = red_grid(n / V16<T>::N);
  if (!ensure_scratch((int)grid + 1, err)) return false;
  k_norm_pass1<T><<<grid, kRedThreads, 0, s>>>(static_cast<const T *>(x), n, g_scratch);
  k_norm_pass2<<<1, kRedThreads, 0, s>>>(g_scratch, (int)grid, g_scratch + grid);
  if (!cuda_ok(cudaGetLastError(), "norm kernel launch", err)) return false;
  return cuda_ok(cudaMemcpyAsync(out, g_scratch + grid, sizeof(double), cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (norm result)", err) &&
         cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (norm)", err);
}

template <typename T>
bool scale_impl(void *x, uint64_t n, double scale, cudaStream_t s, std::string &err) {
  const unsigned grid = red_grid(n / V16<T>::N);
  k_scale<T><<<grid, kRedThreads, 0, s>>>(static_cast<T *>(x), n, (T)scale);
  return cuda_ok(cudaGetLastError(), "scale kernel launch", err);
}

}  // namespace

bool norm_squared(const void *x, uint64_t n_scalars, uint8_t precision, double *out,
                  cudaStream_t s, std::string &err) {
  return precision == 0 ? norm_sq_impl<float>(x, n_scalars, out, s, err)
                        : norm_sq_impl<double>(x, n_scalars, out, s, err);
}

bool scale(void *x, uint64_t n_scalars, uint8_t precision, double factor, cudaStream_t s,
           std::string &err) {
  return precision == 0 ? scale_impl<float>(x, n_scalars, factor, s, err)
                        : scale_impl<double>(x, n_scalars, factor, s, err);
}

}  // namespace cb2

extern "C" {

int cast_cuda_norm_squared(uint64_t dptr, size_t n_elements, uint8_t precision, double *out_norm_sq,
                           char *err_buf, size_t err_buf_len) {
  if (!out_norm_sq) {
    cb2::write_err(err_buf, err_buf_len, "out_norm_sq must not be null");
    return 1;
  }
  std::string err;
  if (!cb2::norm_squared(reinterpret_cast<const void *>(dptr), n_elements, precision, out_norm_sq,
                         nullptr, err)) {
    cb2::write_err(err_buf, err_buf_len, err);
    return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_cuda_scale(uint64_t dptr, size_t n_elements, uint8_t precision, double scale,
                    char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!cb2::scale(reinterpret_cast<void *>(dptr), n_elements, precision, scale, nullptr, err)) {
    cb2::write_err(err_buf, err_buf_len, err);
    return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

}  // extern "C"
