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
#include <type_traits>
#include <vector>

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

// Scratch: partial sums + the final value, one buffer per device, allocated on
// first use and grown on demand (the reference keeps the same kind of
// process-wide scratch, cuda_kernels.cu:203-230).  The mutex serialises users
// of the scratch.  Returns the current device's buffer, or null with a message.
std::mutex g_scratch_mu;
constexpr int kMaxScratchDevices = 64;
double *g_scratch_dev[kMaxScratchDevices] = {};
int g_scratch_len[kMaxScratchDevices] = {};

double *ensure_scratch(int len, std::string &err) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", err)) return nullptr;
  if (dev < 0 || dev >= kMaxScratchDevices) {
    err = "reduction scratch: device index out of range";
    return nullptr;
  }
  double *&p = g_scratch_dev[dev];
  int &have = g_scratch_len[dev];
  if (p && have >= len) return p;
  if (p) cudaFree(p);
  p = nullptr;
  have = 0;
  if (!cuda_ok(cudaMalloc(&p, sizeof(double) * len), "cudaMalloc (norm scratch)", err)) {
    p = nullptr;
    return nullptr;
  }
  have = len;
  return p;
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
  double *const g_scratch = ensure_scratch((int)grid + 1, err);
  if (!g_scratch) return false;
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


// <a|b> partials: (re, im) per block.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_inner_pass1(const T *__restrict__ a,
                                                            const T *__restrict__ b, uint64_t n_amps,
                                                            double *__restrict__ partial) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  const V *av = reinterpret_cast<const V *>(a);
  const V *bv = reinterpret_cast<const V *>(b);
  double re = 0, im = 0;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  for (uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; i < n_amps; i += stride) {
    const V x = av[i], y = bv[i];
    re += (double)x.x * y.x + (double)x.y * y.y;
    im += (double)x.x * y.y - (double)x.y * y.x;
  }
  re = block_sum(re);
  __syncthreads();
  im = block_sum(im);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = re;
    partial[2 * blockIdx.x + 1] = im;
  }
}

// Sums `cols` interleaved columns of `rows` partial rows: out[c] = sum_r p[r*cols + c].
__global__ void __launch_bounds__(kRedThreads) k_sum_columns(const double *__restrict__ p, int rows,
                                                            int cols, double *__restrict__ out) {
  for (int c = blockIdx.x; c < cols; c += gridDim.x) {
    double acc = 0;
    for (int r = threadIdx.x; r < rows; r += kRedThreads) acc += p[(size_t)r * cols + c];
    acc = block_sum(acc);
    if (threadIdx.x == 0) out[c] = acc;
    __syncthreads();
  }
}

constexpr int kMaxPopQubits = 40;

// Per-qubit populations P(q = 1) and the total norm in one pass.  Each thread
// walks 8-amplitude chunks: the chunk's high index bits are constant, so the
// chunk sum is added once per high qubit; the 3 low bits are split per amp.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_populations(const T *__restrict__ x, uint32_t n,
                                                            double *__restrict__ partial) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  const V *xv = reinterpret_cast<const V *>(x);
  const uint64_t n_amps = 1ull << n;
  const uint32_t cb = n < 3 ? n : 3;  // chunk bits
  const uint64_t n_chunks = n_amps >> cb;
  double acc[kMaxPopQubits + 1];
#pragma unroll
  for (int q = 0; q <= kMaxPopQubits; ++q) acc[q] = 0;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  for (uint64_t c = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; c < n_chunks; c += stride) {
    double lo[3] = {0, 0, 0}, tot = 0;
    for (uint32_t j = 0; j < (1u << cb); ++j) {
      const V v = xv[(c << cb) + j];
      const double p = (double)v.x * v.x + (double)v.y * v.y;
      tot += p;
      if (j & 1) lo[0] += p;
      if (j & 2) lo[1] += p;
      if (j & 4) lo[2] += p;
    }
    acc[kMaxPopQubits] += tot;
#pragma unroll
    for (int q = 0; q < 3; ++q) acc[q] += lo[q];
#pragma unroll
    for (int q = 3; q < kMaxPopQubits; ++q)
      if ((uint32_t)q < n && ((c >> (q - 3)) & 1)) acc[q] += tot;
  }
  __shared__ double red[kRedThreads / 32];
#pragma unroll
  for (int q = 0; q <= kMaxPopQubits; ++q) {
    if (q < (int)n || q == kMaxPopQubits) {
      double v = warp_sum(acc[q]);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < kRedThreads / 32; ++w) t += red[w];
        partial[(size_t)blockIdx.x * (kMaxPopQubits + 1) + q] = t;
      }
      __syncthreads();
    }
  }
}

// Marginal probabilities over m measured qubits: per-block bins in shared
// memory (FP64 shared atomics), written as per-block partial rows.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_marginal(const T *__restrict__ x, uint32_t n,
                                                         const uint32_t *__restrict__ measured,
                                                         uint32_t m, double *__restrict__ partial) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  extern __shared__ double bins[];
  const uint32_t nb = 1u << m;
  for (uint32_t i = threadIdx.x; i < nb; i += kRedThreads) bins[i] = 0;
  __shared__ uint32_t mq[16];
  if (threadIdx.x < m) mq[threadIdx.x] = measured[threadIdx.x];
  __syncthreads();
  const V *xv = reinterpret_cast<const V *>(x);
  const uint64_t n_amps = 1ull << n;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  for (uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; i < n_amps; i += stride) {
    const V v = xv[i];
    uint32_t bin = 0;
    for (uint32_t j = 0; j < m; ++j) bin |= (uint32_t)((i >> mq[j]) & 1) << j;
    atomicAdd(&bins[bin], (double)v.x * v.x + (double)v.y * v.y);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nb; i += kRedThreads)
    partial[(size_t)blockIdx.x * nb + i] = bins[i];
}

// A table of powers indexed by a popcount (0 .. kMaxPopQubits), passed to the
// kernels by value (328 bytes of kernel parameters).
struct PopcTable {
  double v[kMaxPopQubits + 1];
};

// Amplitude-damping sums on a qubit mask: per block (T, D) with
// T = sum |a_i|^2 and D = sum |a_i|^2 * w^popc(i & mask), w = 1 - gamma
// (the probability weight of "no jump on any masked qubit"); tab.v[c] = w^c.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_damp_sums(const T *__restrict__ x, uint32_t n,
                                                          uint64_t mask, const PopcTable tab,
                                                          double *__restrict__ partial) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  const V *xv = reinterpret_cast<const V *>(x);
  const uint64_t n_amps = 1ull << n;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  double t = 0, d = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; i < n_amps; i += stride) {
    const V v = xv[i];
    const double p = (double)v.x * v.x + (double)v.y * v.y;
    t += p;
    d += p * tab.v[__popcll(i & mask)];
  }
  t = block_sum(t);
  __syncthreads();
  d = block_sum(d);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = t;
    partial[2 * blockIdx.x + 1] = d;
  }
}

// x_i *= scale * s^popc(i & mask): the no-jump branch of amplitude damping on
// the masked qubits (s = sqrt(1 - gamma)) with its renormalisation folded in.
// tab.v[c] = scale * s^c, computed in FP64 on the host.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_scale_popc(T *__restrict__ x, uint32_t n, uint64_t mask,
                                                           const PopcTable tab) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  V *xv = reinterpret_cast<V *>(x);
  const uint64_t n_amps = 1ull << n;
  const uint64_t stride = (uint64_t)gridDim.x * kRedThreads;
  for (uint64_t i = (uint64_t)blockIdx.x * kRedThreads + threadIdx.x; i < n_amps; i += stride) {
    V v = xv[i];
    const T f = (T)tab.v[__popcll(i & mask)];
    v.x *= f;
    v.y *= f;
    xv[i] = v;
  }
}

template <typename T>
__global__ void k_dm_diag(const T *__restrict__ rho, uint32_t n, double *__restrict__ out) {
  const uint64_t dim = 1ull << n;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (double)rho[2 * (i | (i << n))];
}

template <typename T>
bool inner_impl(const void *a, const void *b, uint32_t n, double *re, double *im, cudaStream_t s,
                std::string &err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const uint64_t amps = 1ull << n;
  const unsigned grid = red_grid(amps);
  double *const g_scratch = ensure_scratch(2 * (int)grid + 2, err);
  if (!g_scratch) return false;
  k_inner_pass1<T><<<grid, kRedThreads, 0, s>>>(static_cast<const T *>(a), static_cast<const T *>(b),
                                                 amps, g_scratch);
  k_sum_columns<<<2, kRedThreads, 0, s>>>(g_scratch, (int)grid, 2, g_scratch + 2 * grid);
  double host[2];
  if (!cuda_ok(cudaGetLastError(), "inner product launch", err) ||
      !cuda_ok(cudaMemcpyAsync(host, g_scratch + 2 * grid, 16, cudaMemcpyDeviceToHost, s),
               "cudaMemcpyAsync (inner product)", err) ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (inner product)", err))
    return false;
  *re = host[0];
  *im = host[1];
  return true;
}

template <typename T>
bool pop_impl(const void *x, uint32_t n, double *p1, double *norm, cudaStream_t s,
              std::string &err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const uint64_t chunks = (1ull << n) >> (n < 3 ? n : 3);
  const unsigned grid = std::min<unsigned>(red_grid(chunks), 2 * sm_count());
  constexpr int W = kMaxPopQubits + 1;
  double *const g_scratch = ensure_scratch(W * ((int)grid + 1), err);
  if (!g_scratch) return false;
  cudaMemsetAsync(g_scratch, 0, sizeof(double) * W * grid, s);
  k_populations<T><<<grid, kRedThreads, 0, s>>>(static_cast<const T *>(x), n, g_scratch);
  k_sum_columns<<<W, kRedThreads, 0, s>>>(g_scratch, (int)grid, W, g_scratch + (size_t)W * grid);
  std::vector<double> host(W);
  if (!cuda_ok(cudaGetLastError(), "populations launch", err) ||
      !cuda_ok(cudaMemcpyAsync(host.data(), g_scratch + (size_t)W * grid, sizeof(double) * W,
                               cudaMemcpyDeviceToHost, s),
               "cudaMemcpyAsync (populations)", err) ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (populations)", err))
    return false;
  for (uint32_t q = 0; q < n; ++q) p1[q] = host[q];
  if (norm) *norm = host[kMaxPopQubits];
  return true;
}

template <typename T>
bool marg_impl(const void *x, uint32_t n, const uint32_t *measured, uint32_t m, double *out,
               cudaStream_t s, std::string &err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const uint32_t nb = 1u << m;
  const unsigned grid = std::min<unsigned>(red_grid(1ull << n), 2 * sm_count());
  const int need = (int)(nb * (grid + 1)) + 16;
  double *const g_scratch = ensure_scratch(need, err);
  if (!g_scratch) return false;
  uint32_t *dq = reinterpret_cast<uint32_t *>(g_scratch + (size_t)nb * (grid + 1));
  if (!cuda_ok(cudaMemcpyAsync(dq, measured, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, s),
               "cudaMemcpyAsync (measured qubits)", err))
    return false;
  k_marginal<T><<<grid, kRedThreads, sizeof(double) * nb, s>>>(static_cast<const T *>(x), n, dq, m,
                                                              g_scratch);
  k_sum_columns<<<std::min<uint32_t>(nb, 1024), kRedThreads, 0, s>>>(g_scratch, (int)grid, (int)nb,
                                                                      g_scratch + (size_t)nb * grid);
  return cuda_ok(cudaGetLastError(), "marginal launch", err) &&
         cuda_ok(cudaMemcpyAsync(out, g_scratch + (size_t)nb * grid, sizeof(double) * nb,
                                 cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (marginal)", err) &&
         cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (marginal)", err);
}

PopcTable powers(double base, double first) {
  PopcTable t;
  double f = first;
  for (int c = 0; c <= kMaxPopQubits; ++c) {
    t.v[c] = f;
    f *= base;
  }
  return t;
}

template <typename T>
bool damp_sums_impl(const void *x, uint32_t n, uint64_t mask, double gamma, double *tot, double *wsum,
                    cudaStream_t s, std::string &err) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned grid = red_grid(1ull << n);
  double *const g_scratch = ensure_scratch(2 * (int)grid + 2, err);
  if (!g_scratch) return false;
  double res[2];
  k_damp_sums<T><<<grid, kRedThreads, 0, s>>>(static_cast<const T *>(x), n, mask,
                                               powers(1.0 - gamma, 1.0), g_scratch);
  k_sum_columns<<<2, kRedThreads, 0, s>>>(g_scratch, (int)grid, 2, g_scratch + 2 * grid);
  if (!cuda_ok(cudaGetLastError(), "damping sums launch", err) ||
      !cuda_ok(cudaMemcpyAsync(res, g_scratch + 2 * grid, 16, cudaMemcpyDeviceToHost, s),
               "cudaMemcpyAsync (damping sums)", err) ||
      !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (damping sums)", err))
    return false;
  *tot = res[0];
  *wsum = res[1];
  return true;
}

template <typename T>
bool scale_popc_impl(void *x, uint32_t n, uint64_t mask, double sfac, double scale, cudaStream_t s,
                     std::string &err) {
  k_scale_popc<T><<<red_grid(1ull << n), kRedThreads, 0, s>>>(static_cast<T *>(x), n, mask,
                                                               powers(sfac, scale));
  return cuda_ok(cudaGetLastError(), "popcount scale launch", err);
}

template <typename T>
bool dm_impl(const void *rho, uint32_t n, double *out, cudaStream_t s, std::string &err) {
  double *d = nullptr;
  const size_t bytes = sizeof(double) << n;
  if (!cuda_ok(cudaMallocAsync(&d, bytes, s), "cudaMallocAsync (dm diagonal)", err)) return false;
  const uint64_t dim = 1ull << n;
  const unsigned grid = (unsigned)std::min<uint64_t>((dim + 255) / 256, 4ull * sm_count());
  k_dm_diag<T><<<grid, 256, 0, s>>>(static_cast<const T *>(rho), n, d);
  const bool ok = cuda_ok(cudaGetLastError(), "dm diagonal launch", err) &&
                  cuda_ok(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, s),
                          "cudaMemcpyAsync (dm diagonal)", err);
  cudaFreeAsync(d, s);
  return ok && cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (dm diagonal)", err);
}

}  // namespace

bool damping_sums(const void *x, uint32_t n, uint8_t precision, uint64_t mask, double gamma,
                  double *tot, double *wsum, cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  if (n == 0 || n > kMaxSvQubits || precision > 1 || !(gamma >= 0.0 && gamma <= 1.0)) {
    err = "damping sums: invalid statevector size, precision or gamma";
    return false;
  }
  return precision == 0 ? damp_sums_impl<float>(x, n, mask, gamma, tot, wsum, s, err)
                        : damp_sums_impl<double>(x, n, mask, gamma, tot, wsum, s, err);
}

bool scale_popc(void *x, uint32_t n, uint8_t precision, uint64_t mask, double sfac, double scale,
                cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  if (n == 0 || n > kMaxSvQubits || precision > 1) {
    err = "popcount scale: invalid statevector size or precision";
    return false;
  }
  return precision == 0 ? scale_popc_impl<float>(x, n, mask, sfac, scale, s, err)
                        : scale_popc_impl<double>(x, n, mask, sfac, scale, s, err);
}

bool norm_squared(const void *x, uint64_t n_scalars, uint8_t precision, double *out,
                  cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  return precision == 0 ? norm_sq_impl<float>(x, n_scalars, out, s, err)
                        : norm_sq_impl<double>(x, n_scalars, out, s, err);
}

bool scale(void *x, uint64_t n_scalars, uint8_t precision, double factor, cudaStream_t s,
           std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  return precision == 0 ? scale_impl<float>(x, n_scalars, factor, s, err)
                        : scale_impl<double>(x, n_scalars, factor, s, err);
}

bool inner_product(const void *a, const void *b, uint32_t n, uint8_t precision, double *re,
                   double *im, cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(a), "first statevector pointer", err) ||
      !aligned16(reinterpret_cast<uint64_t>(b), "second statevector pointer", err))
    return false;
  return precision == 0 ? inner_impl<float>(a, b, n, re, im, s, err)
                        : inner_impl<double>(a, b, n, re, im, s, err);
}

bool qubit_populations(const void *x, uint32_t n, uint8_t precision, double *p1, double *norm,
                       cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  if (n > kMaxPopQubits) {
    err = "populations support at most 40 qubits";
    return false;
  }
  return precision == 0 ? pop_impl<float>(x, n, p1, norm, s, err)
                        : pop_impl<double>(x, n, p1, norm, s, err);
}

bool marginal_probabilities(const void *x, uint32_t n, uint8_t precision, const uint32_t *measured,
                            uint32_t m, double *out, cudaStream_t s, std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(x), "statevector pointer", err)) return false;
  if (m == 0 || m > 12) {
    err = "between 1 and 12 measured qubits are supported";
    return false;
  }
  for (uint32_t j = 0; j < m; ++j)
    if (measured[j] >= n) {
      err = "measured qubit out of range";
      return false;
    }
  return precision == 0 ? marg_impl<float>(x, n, measured, m, out, s, err)
                        : marg_impl<double>(x, n, measured, m, out, s, err);
}

bool dm_populations(const void *rho, uint32_t n, uint8_t precision, double *out, cudaStream_t s,
                    std::string &err) {
  if (!aligned16(reinterpret_cast<uint64_t>(rho), "density-matrix pointer", err)) return false;
  if (2 * n > kMaxSvQubits) {
    err = "density matrix too large";
    return false;
  }
  return precision == 0 ? dm_impl<float>(rho, n, out, s, err) : dm_impl<double>(rho, n, out, s, err);
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
