// On-device shot sampling of a statevector by the inverse CDF.
//
// Replaces the reference's measurement path for CUDA statevectors:
// marginal_probabilities downloads the whole statevector to the host
// (src/simulator/mod.rs:282-291) and batch_sample builds an O(2^n) CDF and
// binary-searches it once per shot (src/simulator/measure.rs:49-76: the
// outcome of a uniform u is the first index whose inclusive prefix sum is
// greater than u, clamped to the last index).  Here the state never leaves HBM.
//
// The CDF is kept in 64-bit fixed point: probability p_i = re^2 + im^2 (FP64,
// each product and the sum rounded separately) becomes
// q_i = round(p_i * 2^62 / T), T the FP64 total.  Integer prefix sums are exact
// and associative, so every parallel order gives the same, monotone CDF; the
// resolution (2^-62 of the total) is far below FP64's rounding of the
// probabilities themselves.  Shot targets are t = floor(u * Q), Q the integer
// total, and the outcome is the first index whose inclusive prefix is > t.
//
//  1. chunk totals: one CTA per chunk of 2^cb amplitudes (cb <= 12) sums its
//     q_i (and its p_i in FP64, for T) - one streaming read of the state.  The
//     first pass assumes T = 1; if the FP64 total is far from 1 it is rerun
//     with the true T (an unnormalised state), so the integers never overflow;
//  2. exact exclusive scans: of the chunk totals (C_c, where chunk c starts in
//     the CDF) and, for seeded sampling, of the shots' exponential spacings;
//  3. assignment: one thread per chunk binary-searches the sorted targets for
//     the chunk's first shot (all chunks in parallel); then one CTA per chunk
//     takes its shots [first_c, first_c+1): a chunk with none exits at once, the
//     others stage q_i in shared memory, form the chunk's inclusive prefix sums
//     and binary-search them per shot.
//
// Sorted uniforms without a sort: with E_0..E_N i.i.d. Exp(1) and
// S_i = E_0 + ... + E_{i-1}, (S_1/S_{N+1}, ..., S_N/S_{N+1}) are distributed as
// the order statistics of N i.i.d. U(0,1) draws (Renyi's representation).  The
// exponentials come from Philox-4x32-10 (shot index as the counter, the seed as
// the key), in 32.32 fixed point so their prefix sums are exact too.
//
// Output: one key per shot, in ascending order of the sampled basis index:
// the index itself, or its bits at the measured qubits compressed to
// positions 0..m-1 (the reference's compress_bits).  Scratch (chunk totals,
// prefixes, spacings, keys) comes from a per-device cache of reused buffers.
#include "../../include/cast_b200.h"
#include "internal.hpp"
#include "philox.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#include <mutex>

namespace cb2 {
namespace {

constexpr int kSmpThreads = 256;
constexpr uint32_t kMaxChunkBits = 12;  // 4096 amplitudes, 16 a thread in the prefix pass
constexpr int kScanThreads = 1024;
constexpr uint32_t kScanPer = 8;  // elements a scan thread sums in order
constexpr uint32_t kMaxMeasured = 64;
constexpr double kFix = 4611686018427387904.0;     // 2^62: probability scale
constexpr double kExpFix = 4294967296.0;           // 2^32: exponential spacings

struct KeyMap {
  uint32_t m;  // 0: the key is the basis index itself
  uint8_t q[kMaxMeasured];
};

__device__ __forceinline__ uint64_t make_key(uint64_t idx, const KeyMap &km) {
  if (km.m == 0) return idx;
  uint64_t key = 0;
  for (uint32_t j = 0; j < km.m; ++j) key |= ((idx >> km.q[j]) & 1ull) << j;
  return key;
}

template <typename V> __device__ __forceinline__ double prob(const V v) {
  // separately rounded products and sum (no fused multiply-add), so a host
  // restatement in IEEE double arithmetic gets the same bits
  return __dadd_rn(__dmul_rn((double)v.x, (double)v.x), __dmul_rn((double)v.y, (double)v.y));
}

__device__ __forceinline__ uint64_t fix(double p, double scale) { return __double2ull_rn(p * scale); }

// Exclusive scan of one uint64 a thread over the block (exact).  `ws` holds NT / 32.
template <int NT>
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane < NT / 32 ? ws[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < NT / 32) ws[lane] = w;
  }
  __syncthreads();
  const uint64_t ex = (warp ? ws[warp - 1] : 0ull) + (inc - v);
  __syncthreads();
  return ex;
}

// Pass 1: integer and FP64 totals of one chunk.
template <typename T>
__global__ void __launch_bounds__(kSmpThreads) k_chunk_totals(const T *__restrict__ x, uint32_t cb,
                                                             double scale, uint64_t *__restrict__ qtot,
                                                             double *__restrict__ ptot) {
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  __shared__ uint64_t wq[kSmpThreads / 32];
  __shared__ double wp[kSmpThreads / 32];
  const uint64_t chunk = blockIdx.x;
  const V *xv = reinterpret_cast<const V *>(x) + (chunk << cb);
  uint64_t q = 0;
  double p = 0.0;
  for (uint32_t i = threadIdx.x; i < (1u << cb); i += kSmpThreads) {
    const double pi = prob(xv[i]);
    q += fix(pi, scale);
    p += pi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    q += __shfl_down_sync(0xffffffffu, q, o);
    p += __shfl_down_sync(0xffffffffu, p, o);
  }
  if ((threadIdx.x & 31) == 0) {
    wq[threadIdx.x >> 5] = q;
    wp[threadIdx.x >> 5] = p;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t a = 0;
    double b = 0.0;
    for (int w = 0; w < kSmpThreads / 32; ++w) {
      a += wq[w];
      b += wp[w];
    }
    qtot[chunk] = a;
    ptot[chunk] = b;
  }
}

// One block: sum of `count` doubles (the FP64 total T).
__global__ void __launch_bounds__(kScanThreads) k_sum_fp(const double *__restrict__ v, uint64_t count,
                                                         double *__restrict__ out) {
  __shared__ double ws[kScanThreads / 32];
  double s = 0.0;
  for (uint64_t i = threadIdx.x; i < count; i += kScanThreads) s += v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < kScanThreads / 32; ++w) a += ws[w];
    *out = a;
  }
}

// Exact exclusive scan of `count` uint64 in tiles of kScanThreads * kScanPer:
// tile totals, one block scanning them in place (and the grand total), then
// each tile rescanned from its offset.
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint64_t *__restrict__ in,
                                                             uint64_t count,
                                                             uint64_t *__restrict__ tile_total) {
  __shared__ uint64_t ws[kScanThreads / 32];
  const uint64_t base = ((uint64_t)blockIdx.x * kScanThreads + threadIdx.x) * kScanPer;
  uint64_t s = 0;
  for (uint32_t j = 0; j < kScanPer; ++j)
    if (base + j < count) s += in[base + j];
  const uint64_t ex = block_exclusive_scan<kScanThreads>(s, ws);
  if (threadIdx.x == kScanThreads - 1) tile_total[blockIdx.x] = ex + s;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_small(uint64_t *__restrict__ v, uint64_t count,
                                                             uint64_t *__restrict__ grand) {
  __shared__ uint64_t ws[kScanThreads / 32];
  const uint64_t per = (count + kScanThreads - 1) / kScanThreads;
  const uint64_t base = (uint64_t)threadIdx.x * per;
  uint64_t s = 0;
  for (uint64_t j = 0; j < per; ++j)
    if (base + j < count) s += v[base + j];
  const uint64_t ex = block_exclusive_scan<kScanThreads>(s, ws);
  uint64_t run = ex;
  for (uint64_t j = 0; j < per; ++j)
    if (base + j < count) {
      const uint64_t y = v[base + j];
      v[base + j] = run;
      run += y;
    }
  if (threadIdx.x == kScanThreads - 1) *grand = ex + s;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint64_t *__restrict__ in,
                                                             uint64_t count,
                                                             const uint64_t *__restrict__ tile_off,
                                                             uint64_t *__restrict__ out) {
  __shared__ uint64_t ws[kScanThreads / 32];
  const uint64_t base = ((uint64_t)blockIdx.x * kScanThreads + threadIdx.x) * kScanPer;
  uint64_t s = 0;
  for (uint32_t j = 0; j < kScanPer; ++j)
    if (base + j < count) s += in[base + j];
  uint64_t run = tile_off[blockIdx.x] + block_exclusive_scan<kScanThreads>(s, ws);
  for (uint32_t j = 0; j < kScanPer; ++j)
    if (base + j < count) {
      const uint64_t y = in[base + j];
      out[base + j] = run;
      run += y;
    }
}

// E_i = -log(1 - u_i) in 32.32 fixed point, u_i in [0, 1) from Philox with the
// counter (i_lo, i_hi, 0x5a3b1e5, 0) and the seed as the key.
__global__ void k_exponentials(uint64_t seed, uint64_t count, uint64_t *__restrict__ e) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0x5a3b1e5u, 0u};
    philox4x32_10(x, (uint32_t)seed, (uint32_t)(seed >> 32));
    e[i] = __double2ull_rn(-log(1.0 - philox_unit(x)) * kExpFix);
  }
}

// Where shot i lands in the integer CDF: t_i = floor(f_i * Q) with
// f_i = S_{i+1} / S_{N+1} (seeded) or the caller's u_i.  Non-decreasing in i.
// Q and S_{N+1} are read on the device from the scans' grand totals
// (`resolve`), so no host round trip sits between the scans and the searches.
struct Targets {
  const uint64_t *spacing;  // exclusive prefix of the N+1 spacings (seeded), or null
  const double *u;          // sorted uniforms (caller-given), or null
  const uint64_t *grand;    // [0] Q, [1] spacing total
  uint64_t spacing_total;
  double q_total;  // Q as a double
  __device__ __forceinline__ void resolve() {
    q_total = (double)grand[0];
    spacing_total = grand[1];
  }
  __device__ __forceinline__ uint64_t operator()(uint64_t i) const {
    const double f = spacing ? __ddiv_rn((double)spacing[i + 1], (double)spacing_total) : u[i];
    return __double2ull_rd(__dmul_rn(f, q_total));
  }
};

// Status of one sampling pass, written to grand[3] before the searches run:
// 0 go on, 1 the FP64 total is zero or not finite, 2 the total is far from 1
// (the integer totals may have overflowed: the host reruns the pass with the
// true total as scale), 3 the integer CDF or the spacings sum to zero.  The
// search and assignment kernels return at once unless it is 0.
__global__ void k_check(uint64_t *__restrict__ grand, int seeded, int need_range) {
  if (threadIdx.x || blockIdx.x) return;
  const double t = __longlong_as_double((long long)grand[2]);
  uint64_t st = 0;
  if (!(t > 0.0) || !isfinite(t)) st = 1;
  else if (need_range && !(t > 0.5 && t < 2.0)) st = 2;
  else if (grand[0] == 0 || (seeded && grand[1] == 0)) st = 3;
  grand[3] = st;
}

// Shot ranges: first[c] = the first shot whose target is >= the start of chunk c
// (first[0] = 0, first[n_chunks] = n_shots), one thread a chunk, all chunks'
// binary searches in parallel; chunk c takes shots first[c] .. first[c+1] - 1.
__global__ void k_chunk_first_shot(const uint64_t *__restrict__ start, uint64_t n_chunks,
                                   Targets tg, uint64_t n_shots, uint64_t *__restrict__ first) {
  if (tg.grand[3] != 0) return;
  tg.resolve();
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c <= n_chunks;
       c += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t a = 0, b = n_shots;
    if (c == 0) {
      b = 0;
    } else if (c == n_chunks) {
      a = n_shots;
    } else {
      const uint64_t bound = start[c];
      while (a < b) {
        const uint64_t mid = a + (b - a) / 2;
        if (tg(mid) < bound) a = mid + 1;
        else b = mid;
      }
    }
    first[c] = a;
  }
}

// Pass 3.
template <typename T>
__global__ void __launch_bounds__(kSmpThreads) k_sample_assign(
    const T *__restrict__ x, uint32_t cb, const uint64_t *__restrict__ start,
    const uint64_t *__restrict__ first, Targets tg, double scale,
    const __grid_constant__ KeyMap km, uint64_t *__restrict__ out) {
  if (tg.grand[3] != 0) return;
  tg.resolve();
  using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  // one padding slot after every 16: a thread's run of 16 starts 17 slots after
  // its neighbour's, so the runs of a warp sit in different banks
  __shared__ uint64_t q[(1u << kMaxChunkBits) + (1u << kMaxChunkBits) / 16];
  __shared__ uint64_t ws[kSmpThreads / 32];
  const uint64_t chunk = blockIdx.x;
  const uint64_t lo = first[chunk], hi = first[chunk + 1];
  if (lo >= hi) return;
  const uint32_t c = 1u << cb;
  const uint32_t nt = c < (uint32_t)kSmpThreads ? c : (uint32_t)kSmpThreads;
  const uint32_t per = c / nt;
  const V *xv = reinterpret_cast<const V *>(x) + (chunk << cb);
  for (uint32_t i = threadIdx.x; i < c; i += kSmpThreads) q[i + (i >> 4)] = fix(prob(xv[i]), scale);
  __syncthreads();
  uint64_t s = 0;
  if (threadIdx.x < nt)
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t i = threadIdx.x * per + j;
      s += q[i + (i >> 4)];
    }
  uint64_t run = start[chunk] + block_exclusive_scan<kSmpThreads>(s, ws);
  if (threadIdx.x < nt)
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t i = threadIdx.x * per + j;
      run += q[i + (i >> 4)];
      q[i + (i >> 4)] = run;  // inclusive CDF value of amplitude i
    }
  __syncthreads();
  for (uint64_t i = lo + threadIdx.x; i < hi; i += kSmpThreads) {
    const uint64_t t = tg(i);
    uint32_t a = 0, b = c;  // first j with cdf[j] > t
    while (a < b) {
      const uint32_t mid = (a + b) >> 1;
      if (q[mid + (mid >> 4)] <= t) a = mid + 1;
      else b = mid;
    }
    if (a >= c) a = c - 1;
    out[i] = make_key((chunk << cb) + a, km);
  }
}

// Scratch buffers, per device, kept for the process's lifetime and reused: a
// call takes the smallest free buffer that fits (or allocates one, rounded up
// to 32 MiB) and returns it when done, so concurrent callers each hold their
// own and a steady stream of calls allocates nothing.  Stream-ordered
// allocation from the default pool hands the memory back at every synchronize
// and re-maps it on the next call: 1M shots from a 30-qubit complex128 state
// took 6.0-6.3 ms with spikes to 25 ms (28-74 ms on another box) that way,
// 5.5-5.7 ms with these buffers.
struct ScratchCache {
  std::mutex mu;
  std::vector<std::pair<int, std::pair<char *, size_t>>> free;  // (device, (buffer, bytes))
};
ScratchCache &scratch_cache() {
  static ScratchCache c;
  return c;
}

bool take_scratch(size_t bytes, char **out, size_t *got, std::string &err) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", err)) return false;
  ScratchCache &c = scratch_cache();
  {
    std::lock_guard<std::mutex> lock(c.mu);
    size_t best = c.free.size();
    for (size_t i = 0; i < c.free.size(); ++i)
      if (c.free[i].first == dev && c.free[i].second.second >= bytes &&
          (best == c.free.size() || c.free[i].second.second < c.free[best].second.second))
        best = i;
    if (best < c.free.size()) {
      *out = c.free[best].second.first;
      *got = c.free[best].second.second;
      c.free.erase(c.free.begin() + (std::ptrdiff_t)best);
      return true;
    }
  }
  const size_t unit = size_t(32) << 20;
  *got = (bytes + unit - 1) / unit * unit;
  return cuda_ok(cudaMalloc((void **)out, *got), "cudaMalloc (sampling scratch)", err);
}

void give_scratch(char *p, size_t bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  ScratchCache &c = scratch_cache();
  std::lock_guard<std::mutex> lock(c.mu);
  c.free.push_back({dev, {p, bytes}});
}

template <typename T>
bool sample_impl(const void *sv, uint32_t n, uint64_t n_shots, bool seeded, uint64_t seed,
                 const double *host_u, const KeyMap &km, uint64_t *host_out, cudaStream_t s,
                 std::string &err) {
  const uint32_t cb = n < kMaxChunkBits ? n : kMaxChunkBits;
  const uint64_t n_chunks = 1ull << (n - cb);
  const uint64_t n_sp = seeded ? n_shots + 1 : 0;
  const uint64_t tile = (uint64_t)kScanThreads * kScanPer;
  const uint64_t tiles_c = (n_chunks + tile - 1) / tile, tiles_s = (n_sp + tile - 1) / tile;
  // 8-byte slots: chunk totals (int, FP64), chunk starts, tile totals (both
  // scans), grand totals, spacings (raw and scanned) or uniforms, keys
  const uint64_t slots = 4 * n_chunks + 1 + tiles_c + tiles_s + 4 + (seeded ? 2 * n_sp : n_shots) + n_shots;
  char *scratch = nullptr;
  size_t scratch_bytes = 0;
  if (!take_scratch(slots * 8, &scratch, &scratch_bytes, err)) return false;
  uint64_t *qtot = reinterpret_cast<uint64_t *>(scratch);
  double *ptot = reinterpret_cast<double *>(qtot + n_chunks);
  uint64_t *start = qtot + 2 * n_chunks;
  uint64_t *first = start + n_chunks;  // n_chunks + 1 entries
  uint64_t *tt_c = first + n_chunks + 1;
  uint64_t *tt_s = tt_c + tiles_c;
  uint64_t *grand = tt_s + tiles_s;  // [0] Q, [1] spacing total, [2] FP64 T (bits)
  uint64_t *sp_raw = grand + 4;
  uint64_t *sp = sp_raw + n_sp;
  double *u_dev = reinterpret_cast<double *>(sp_raw);
  uint64_t *keys = sp_raw + (seeded ? 2 * n_sp : n_shots);
  const T *x = static_cast<const T *>(sv);
  const Targets tg{seeded ? sp : nullptr, seeded ? nullptr : u_dev, grand, 0, 0.0};
  std::string e2;
  bool ok = true;
  double scale = kFix;
  // A normalised state takes one pass with no host round trip before the final
  // copy: the totals, scans, status check, searches and assignment are queued
  // back to back and the host reads the status with the keys.  Only a state
  // whose total is far from 1 takes a second pass, scaled by its true total.
  for (int attempt = 0; attempt < 2 && ok; ++attempt) {
    k_chunk_totals<T><<<(unsigned)n_chunks, kSmpThreads, 0, s>>>(x, cb, scale, qtot, ptot);
    k_sum_fp<<<1, kScanThreads, 0, s>>>(ptot, n_chunks, reinterpret_cast<double *>(grand + 2));
    k_scan_tiles<<<(unsigned)tiles_c, kScanThreads, 0, s>>>(qtot, n_chunks, tt_c);
    k_scan_small<<<1, kScanThreads, 0, s>>>(tt_c, tiles_c, grand);
    k_scan_apply<<<(unsigned)tiles_c, kScanThreads, 0, s>>>(qtot, n_chunks, tt_c, start);
    if (attempt == 0) {  // the spacings or uniforms do not depend on the scale
      if (seeded) {
        const unsigned eg = (unsigned)std::min<uint64_t>((n_sp + 255) / 256, 16ull * sm_count());
        k_exponentials<<<eg, 256, 0, s>>>(seed, n_sp, sp_raw);
        k_scan_tiles<<<(unsigned)tiles_s, kScanThreads, 0, s>>>(sp_raw, n_sp, tt_s);
        k_scan_small<<<1, kScanThreads, 0, s>>>(tt_s, tiles_s, grand + 1);
        k_scan_apply<<<(unsigned)tiles_s, kScanThreads, 0, s>>>(sp_raw, n_sp, tt_s, sp);
      } else {
        ok = cuda_ok(cudaMemcpyAsync(u_dev, host_u, n_shots * 8, cudaMemcpyHostToDevice, s),
                     "cudaMemcpyAsync (uniforms)", err);
        if (!ok) break;
      }
    }
    k_check<<<1, 32, 0, s>>>(grand, seeded ? 1 : 0, attempt == 0 ? 1 : 0);
    const unsigned fg = (unsigned)std::min<uint64_t>((n_chunks + 256) / 256, 16ull * sm_count());
    k_chunk_first_shot<<<fg, 256, 0, s>>>(start, n_chunks, tg, n_shots, first);
    k_sample_assign<T><<<(unsigned)n_chunks, kSmpThreads, 0, s>>>(x, cb, start, first, tg, scale, km,
                                                                   keys);
    uint64_t g[4] = {0, 0, 0, 0};
    ok = cuda_ok(cudaGetLastError(), "sampling launch", err) &&
         cuda_ok(cudaMemcpyAsync(host_out, keys, n_shots * 8, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (sampled keys)", err) &&
         cuda_ok(cudaMemcpyAsync(g, grand, sizeof(g), cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (sampling status)", err) &&
         cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (sampling)", err);
    if (!ok) break;
    if (g[3] == 0) break;
    double total;
    std::memcpy(&total, &g[2], sizeof(total));
    if (g[3] == 1) {
      err = "cannot sample a statevector whose total probability is zero or not finite";
      ok = false;
    } else if (g[3] == 3) {
      err = "sampling: the integer CDF or the spacings summed to zero";
      ok = false;
    } else if (attempt == 0) {
      scale = kFix / total;  // unnormalised state: scale to Q ~ 2^62
    } else {
      err = "sampling: the rescaled pass did not settle";
      ok = false;
    }
  }
  // the buffer goes back only once the stream is done with it
  const bool synced = cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (sampling)", e2);
  if (synced) give_scratch(scratch, scratch_bytes);
  if (ok && !synced) err = e2;
  return ok && synced;
}

bool sample_entry(uint64_t dptr, uint32_t n, uint8_t precision, uint64_t n_shots, bool seeded,
                  uint64_t seed, const double *host_u, const uint32_t *measured, uint32_t n_measured,
                  uint64_t *out, void *stream, std::string &err) {
  if (!dptr || (n_shots && !out)) {
    err = "statevector and output must not be null";
    return false;
  }
  if (!aligned16(dptr, "statevector pointer", err)) return false;
  if (precision > 1 || n == 0 || n > 36) {
    err = "sampling supports F32 / F64 statevectors of 1..36 qubits";
    return false;
  }
  if (n_shots > (1ull << 30)) {
    err = "at most 2^30 shots per call";
    return false;
  }
  KeyMap km{};
  if (n_measured > 0) {
    if (!measured || n_measured > n || n_measured > kMaxMeasured) {
      err = "measured qubits: between 1 and n distinct qubits (or none for full basis indices)";
      return false;
    }
    uint64_t seen = 0;
    for (uint32_t j = 0; j < n_measured; ++j) {
      if (measured[j] >= n || ((seen >> measured[j]) & 1)) {
        err = "measured qubits must be distinct and below the qubit count";
        return false;
      }
      seen |= 1ull << measured[j];
      km.q[j] = (uint8_t)measured[j];
    }
    km.m = n_measured;
  }
  if (!seeded && n_shots) {
    if (!host_u) {
      err = "uniforms must not be null";
      return false;
    }
    for (uint64_t i = 0; i < n_shots; ++i)
      if (!(host_u[i] >= 0.0 && host_u[i] < 1.0) || (i && host_u[i] < host_u[i - 1])) {
        err = "uniforms must be non-decreasing and in [0, 1)";
        return false;
      }
  }
  if (n_shots == 0) return true;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return precision == 0
             ? sample_impl<float>(reinterpret_cast<const void *>(dptr), n, n_shots, seeded, seed,
                                  host_u, km, out, s, err)
             : sample_impl<double>(reinterpret_cast<const void *>(dptr), n, n_shots, seeded, seed,
                                   host_u, km, out, s, err);
}

}  // namespace
}  // namespace cb2

extern "C" {

int cast_b200_sample(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t n_shots,
                     uint64_t seed, const uint32_t *measured, uint32_t n_measured,
                     uint64_t *out_keys, void *stream, char *err_buf, size_t err_buf_len) {
  std::string err;
  try {
    if (!cb2::sample_entry(sv_dptr, n_qubits, precision, n_shots, true, seed, nullptr, measured,
                           n_measured, out_keys, stream, err)) {
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
  } catch (const std::exception &ex) {
    cb2::write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_sample_at(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                        const double *sorted_uniforms, uint64_t n_shots, const uint32_t *measured,
                        uint32_t n_measured, uint64_t *out_keys, void *stream, char *err_buf,
                        size_t err_buf_len) {
  std::string err;
  try {
    if (!cb2::sample_entry(sv_dptr, n_qubits, precision, n_shots, false, 0, sorted_uniforms,
                           measured, n_measured, out_keys, stream, err)) {
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
  } catch (const std::exception &ex) {
    cb2::write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

}  // extern "C"
