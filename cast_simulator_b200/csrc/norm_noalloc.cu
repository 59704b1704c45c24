// Allocation-free variant of the statevector norm^2 reduction.
//
// cast_cuda_norm_squared keeps its per-block partial sums in a device buffer
// that the library allocates with cudaMalloc on first use.  Some callers
// cannot let a library allocate device memory: applications whose device
// memory is owned by a pool or arena that must account for every byte (an
// allocation behind its back can push the pool past its budget), and hosts
// that forbid allocations once they are running (cudaMalloc and cudaFree may
// synchronise the whole device, which stalls every other stream of a
// latency-bound service).  This entry point serves them: its scratch is a
// file-scope __device__ array of fixed size, created when the library is
// loaded onto a device and held until the process exits (kNoAllocPartials + 1
// doubles, about 1 MiB, on every GPU that loads the library).  It calls no
// cudaMalloc / cudaFree and no allocating library routine.
//
// Each block of the first pass reduces a fixed chunk of 256 threads x 64
// 128-bit vectors and writes one partial; the second pass folds the partials
// into the last slot.  The partial count therefore grows with the input, and
// inputs needing more than kNoAllocPartials partials are rejected.  Every slot
// that is read is written earlier in the same call, so nothing needs clearing
// between calls; but all calls share the one array, so two calls whose kernels
// overlap on the GPU (different streams, no ordering between them) race on it.
#include "../../include/cast_b200.h"
#include "internal.hpp"

#include <cuda.h>

#include <mutex>

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaVecPerThread = 64;
constexpr uint64_t kNaVecPerBlock = (uint64_t)kNaThreads * kNaVecPerThread;  // 16384 vectors
constexpr uint64_t kNoAllocPartials = 1ull << 17;
constexpr int kMaxDevices = 64;

// The scratch: partials[0 .. blocks) and the result at partials[kNoAllocPartials].
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPartials + 1];

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int THREADS> __device__ __forceinline__ double na_block_sum(double v) {
  __shared__ double part[THREADS / 32];
  v = na_warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  v = threadIdx.x < THREADS / 32 ? part[threadIdx.x] : 0.0;
  if (threadIdx.x < 32) v = na_warp_sum(v);
  return v;
}

__device__ __forceinline__ double na_sq(float4 v) {
  return (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
}
__device__ __forceinline__ double na_sq(double2 v) { return v.x * v.x + v.y * v.y; }

// Pass 1: block b sums vectors [b * kNaVecPerBlock, (b+1) * kNaVecPerBlock) and
// the scalar tail (block 0), writing partials[b].
template <typename T>
__global__ void __launch_bounds__(kNaThreads) k_na_pass1(const T *__restrict__ x, uint64_t n,
                                                         double *__restrict__ partials) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  constexpr uint64_t N = sizeof(V) / sizeof(T);
  const V *xv = reinterpret_cast<const V *>(x);
  const uint64_t nv = n / N;
  const uint64_t begin = (uint64_t)blockIdx.x * kNaVecPerBlock;
  const uint64_t end = begin + kNaVecPerBlock < nv ? begin + kNaVecPerBlock : nv;
  double a0 = 0, a1 = 0;
  uint64_t i = begin + threadIdx.x;
  for (; i + kNaThreads < end; i += 2 * kNaThreads) {
    a0 += na_sq(xv[i]);
    a1 += na_sq(xv[i + kNaThreads]);
  }
  if (i < end) a0 += na_sq(xv[i]);
  double acc = a0 + a1;
  if (blockIdx.x == 0 && threadIdx.x < n - nv * N) {
    const double t = (double)x[nv * N + threadIdx.x];
    acc += t * t;
  }
  acc = na_block_sum<kNaThreads>(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// Pass 2: partials[kNoAllocPartials] = sum of partials[0 .. count).
__global__ void __launch_bounds__(1024) k_na_pass2(double *__restrict__ partials, uint32_t count) {
  double acc = 0;
  for (uint32_t i = threadIdx.x; i < count; i += 1024) acc += partials[i];
  acc = na_block_sum<1024>(acc);
  if (threadIdx.x == 0) partials[kNoAllocPartials] = acc;
}

// Device address of g_noalloc_scratch.  In host code the symbol is only a
// host-side handle, so the address is looked up with cudaGetSymbolAddress, with
// the device current, once per device: the set-up step, taken by the first
// call on each device.  The address belongs to the device's context; a
// cudaDeviceReset destroys that context and the next one may load the array
// elsewhere.  So each entry also records the unique ID of the context it was
// resolved in, and a call that finds a different context (after a reset)
// resolves the address again.  The driver calls go through
// cudaGetDriverEntryPoint, so the library needs no link against libcuda.
using PfnCtxGetCurrent = CUresult (*)(CUcontext *);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long *);

struct ScratchEntry {
  double *addr = nullptr;
  unsigned long long ctx_id = 0;
};

std::mutex g_na_mu;
ScratchEntry g_na_table[kMaxDevices];
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;

// The unique ID of the calling thread's current context, or 0 when there is
// none (or the driver cannot tell).
unsigned long long current_context_id() {
  if (!g_ctx_get_current || !g_ctx_get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

bool scratch_address(double **out, std::string &err) {
  int dev = 0;
  if (!cb2::cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", err)) return false;
  if (dev < 0 || dev >= kMaxDevices) {
    err = "device index out of range for the allocation-free scratch table";
    return false;
  }
  std::lock_guard<std::mutex> lock(g_na_mu);
  if (!g_ctx_get_current || !g_ctx_get_id) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSuccess, q2 = q1;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
      g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f2);
    }
    (void)cudaGetLastError();
  }
  ScratchEntry &e = g_na_table[dev];
  if (e.addr) {
    const unsigned long long id = current_context_id();
    if (id != 0 && id == e.ctx_id) {
      *out = e.addr;
      return true;
    }
  }
  void *p = nullptr;
  if (!cb2::cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                    "cudaGetSymbolAddress (allocation-free scratch)", err))
    return false;
  e.addr = static_cast<double *>(p);
  e.ctx_id = current_context_id();  // 0 (never matches): resolve again on every call
  *out = e.addr;
  return true;
}

template <typename T>
bool norm_noalloc(const void *x, uint64_t n, double *out, cudaStream_t s, std::string &err) {
  constexpr uint64_t N = sizeof(T) == 8 ? 2 : 4;
  const uint64_t nv = n / N;
  const uint64_t blocks = nv == 0 ? 1 : (nv + kNaVecPerBlock - 1) / kNaVecPerBlock;
  if (blocks > kNoAllocPartials) {
    err = "allocation-free norm: " + std::to_string(n) + " scalars exceed the maximum of " +
          std::to_string(kNoAllocPartials * kNaVecPerBlock * N) +
          " scalars that its fixed scratch supports";
    return false;
  }
  double *scratch = nullptr;
  if (!scratch_address(&scratch, err)) return false;
  k_na_pass1<T><<<(unsigned)blocks, kNaThreads, 0, s>>>(static_cast<const T *>(x), n, scratch);
  k_na_pass2<<<1, 1024, 0, s>>>(scratch, (uint32_t)blocks);
  return cb2::cuda_ok(cudaGetLastError(), "allocation-free norm launch", err) &&
         cb2::cuda_ok(cudaMemcpyAsync(out, scratch + kNoAllocPartials, sizeof(double),
                                      cudaMemcpyDeviceToHost, s),
                      "cudaMemcpyAsync (allocation-free norm result)", err) &&
         cb2::cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (allocation-free norm)",
                      err);
}

}  // namespace

extern "C" int cast_b200_norm_squared_noalloc(uint64_t dptr, size_t n_elements, uint8_t precision,
                                              double *out_norm_sq, void *stream, char *err_buf,
                                              size_t err_buf_len) {
  if (!dptr || !out_norm_sq) {
    cb2::write_err(err_buf, err_buf_len, "dptr and out_norm_sq must not be null");
    return 1;
  }
  if (precision > 1) {
    cb2::write_err(err_buf, err_buf_len, "precision must be 0 (F32) or 1 (F64)");
    return 1;
  }
  std::string err;
  if (!cb2::aligned16(dptr, "dptr", err)) {
    cb2::write_err(err_buf, err_buf_len, err);
    return 1;
  }
  const bool ok =
      precision == 0
          ? norm_noalloc<float>(reinterpret_cast<const void *>(dptr), n_elements, out_norm_sq,
                                static_cast<cudaStream_t>(stream), err)
          : norm_noalloc<double>(reinterpret_cast<const void *>(dptr), n_elements, out_norm_sq,
                                 static_cast<cudaStream_t>(stream), err);
  if (!ok) {
    cb2::write_err(err_buf, err_buf_len, err);
    return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}
