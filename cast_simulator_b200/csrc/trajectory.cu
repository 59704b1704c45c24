// Batched Monte-Carlo quantum-jump trajectories in one persistent kernel.
//
// Replaces the reference's ensemble simulation (src/simulator/trajectory.rs:
// simulate_ensemble at :180-265 branches deterministically on fixed weights
// p_i and launches one kernel per gate per member, syncing with the host at
// every noisy gate) with quantum-jump trajectories sampled on the device:
//
//  * one CTA (512 or 1024 threads) owns one trajectory at a time; its 2^n
//    complex64 statevector lives in a per-CTA slice of a workspace in global
//    memory (148 CTAs x 512 KiB = 74 MiB at 16 qubits, resident in the 126 MB
//    L2); the CTA loops over trajectories blockIdx.x, blockIdx.x + gridDim.x, ...
//  * GATE ops are fused unitary blocks (k <= 4) applied in place;
//  * ERR ops are state-independent Pauli errors (depolarizing): a Philox draw
//    decides; when one fires, the Pauli propagated to the end of its fused
//    block (U P U^dagger, precomputed on the host) is applied as a gate;
//  * DAMP ops are amplitude damping on a set of qubits.  The no-jump branch has
//    probability D/T with T = sum |a_i|^2 and D = sum |a_i|^2 (1-g)^popc(i&mask),
//    both FP64 sums computed by the preceding gate pass as it stores; on a
//    no-jump draw the diagonal prod_q K0_q and the 1/sqrt(D) renormalisation are
//    folded into the next pass's loads.  Otherwise the jump pattern is sampled
//    exactly, qubit by qubit, conditioned on at least one jump;
//  * CHAN ops are general single-qubit channels: FP64 branch norms
//    ||K_j psi||^2, one draw, K_j / sqrt(p_j) applied.
// At the end each trajectory writes <Z_q> for every qubit and one measured
// bitstring sampled from |psi|^2.  Branch sums, renormalisation factors and the
// final reductions are FP64; amplitudes and gate arithmetic are FP32.
#include "../../include/cast_b200.h"
#include "internal.hpp"
#include "philox.cuh"

#include <algorithm>
#include <cmath>
#include <exception>
#include <map>
#include <mutex>
#include <vector>

namespace {

using cb2::cuda_ok;

// A CTA has 512 or 1024 threads (the kernel is instantiated for both).
constexpr int kTMinThreads = 512, kTMaxThreads = 1024;
constexpr uint32_t kTrajMaxQubits = 22;
constexpr uint32_t kTrajMaxGate = 4;

enum : uint32_t { T_GATE = 0, T_ERR = 1, T_DAMP = 2, T_CHAN = 3 };

struct TOp {
  uint32_t type;
  uint32_t k;
  uint32_t q[kTrajMaxGate];
  uint32_t mat;    // complex offset into the matrix pool
  uint32_t nk;     // CHAN: number of Kraus operators (<= 4)
  uint32_t mask;   // DAMP: qubits
  uint32_t stats;  // GATE: accumulate (T, D) for the DAMP op that follows
  uint32_t nerr;   // GATE: number of ERR ops that directly follow it
  uint32_t smask;  // GATE stats: damping mask of that op
  float prob;      // ERR: firing probability
  float gamma;     // DAMP: damping rate
  float sgamma;    // GATE stats: damping rate of that op
};

struct TRun {  // device-resident, rewritten before each launch
  uint32_t n_traj;
  uint32_t first;  // index of the first trajectory (its Philox stream), for ranges
  uint64_t seed;
};

// Philox-4x32-10 (philox.cuh): counter (event, 0, trajectory, 0x5eed5eed),
// key = the 64-bit seed.
__device__ __forceinline__ double philox_uniform(uint64_t seed, uint32_t traj, uint32_t event) {
  uint32_t x[4] = {event, 0u, traj, 0x5eed5eedu};
  cb2::philox4x32_10(x, (uint32_t)seed, (uint32_t)(seed >> 32));
  return cb2::philox_unit(x);
}

struct Shared {
  double red[3][kTMaxThreads / 32];
  double vals[4];
  float dtab[kTrajMaxQubits + 1];  // pending diagonal: scale * s^popc
  double stab[kTrajMaxQubits + 1]; // damping weights (1 - g)^popc for the sums
  uint32_t pmask;
  int pend;
};

__device__ __forceinline__ float2 cmul_add(float2 m, float2 x, float2 acc) {
  acc.x = fmaf(m.x, x.x, acc.x);
  acc.x = fmaf(-m.y, x.y, acc.x);
  acc.y = fmaf(m.x, x.y, acc.y);
  acc.y = fmaf(m.y, x.x, acc.y);
  return acc;
}

// The device side of one trajectory, for CTAs of NT threads.  512-thread CTAs
// get 128 registers a thread, so the fused gates run without spills (the passes
// of small and HBM-sized states are bound by instruction issue); 1024-thread
// CTAs keep twice the loads in flight, which is what the L2-resident states of
// 15 to 17 qubits need.
template <int NT>
struct Traj {
  static constexpr int kTThreads = NT;
  static constexpr uint32_t kTLogThreads = NT == 1024 ? 10 : 9;

  // Block sum of up to three doubles; every thread gets the results.
  static __device__ void block_sum3(Shared &S, double &a, double &b, double &c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
      c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      S.red[0][w] = a;
      S.red[1][w] = b;
      S.red[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double x = 0, y = 0, z = 0;
      for (int i = 0; i < kTThreads / 32; ++i) {
        x += S.red[0][i];
        y += S.red[1][i];
        z += S.red[2][i];
      }
      S.vals[0] = x;
      S.vals[1] = y;
      S.vals[2] = z;
    }
    __syncthreads();
    a = S.vals[0];
    b = S.vals[1];
    c = S.vals[2];
    __syncthreads();
  }

  static __device__ void fill_stab(Shared &S, double g) {
    if (threadIdx.x == 0) {
      double f = 1.0;
      for (uint32_t c = 0; c <= kTrajMaxQubits; ++c) {
        S.stab[c] = f;
        f *= 1.0 - g;
      }
    }
    __syncthreads();
  }

  static __device__ __forceinline__ float2 pend_load(const float2 *sv, uint32_t i, const Shared &S) {
    float2 v = sv[i];
    if (S.pend) {
      const float f = S.dtab[__popc(i & S.pmask)];
      v.x *= f;
      v.y *= f;
    }
    return v;
  }

  // Fused-gate pass (k = K).  PEND: the pending diagonal (scale * s^popc(i & pmask))
  // is applied to every loaded amplitude.  With op.stats the pass also sums, over
  // its outputs, t += |o|^2 and d += |o|^2 (1-g)^popc(i & smask) for the damping op
  // that follows.
  //
  // k = 1 gates take two groups a thread, so every matrix load serves both.
  template <int K>
  static constexpr int groups_per_thread() { return K == 1 ? 2 : 1; }

  template <int K, bool PEND>
  static __device__ __noinline__ void gate_pass(float2 *sv, uint32_t n, const TOp &op, const float2 *M,
                                         const Shared &S, double &t, double &d) {
    constexpr int D = 1 << K;
    constexpr int U = groups_per_thread<K>();
    uint32_t lo[K];
#pragma unroll
    for (int b = 0; b < K; ++b) lo[b] = (1u << op.q[b]) - 1;
    const uint32_t ng = 1u << (n - K);
    const bool stats = op.stats != 0;
    const uint32_t smask = op.smask;
    const uint32_t pmask = S.pmask;
    double lt = 0, ld = 0;
    for (uint32_t g0 = threadIdx.x; g0 < ng; g0 += kTThreads * U) {
      uint32_t base[U];
      float2 x[U][D];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t g = g0 + u * kTThreads;
        uint32_t bb = g < ng ? g : 0;
#pragma unroll
        for (int b = 0; b < K; ++b) bb = ((bb & ~lo[b]) << 1) | (bb & lo[b]);
        base[u] = bb;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          uint32_t o = bb;
#pragma unroll
          for (int b = 0; b < K; ++b)
            if ((a >> b) & 1) o += lo[b] + 1;
          float2 v = make_float2(0.f, 0.f);
          if (g < ng) v = sv[o];
          if (PEND) {
            const float f = S.dtab[__popc(o & pmask)];
            v.x *= f;
            v.y *= f;
          }
          x[u][a] = v;
        }
      }
#pragma unroll
      for (int r = 0; r < D; ++r) {
        float2 acc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) acc[u] = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < D; ++c) {
          const float2 m = M[r * D + c];
#pragma unroll
          for (int u = 0; u < U; ++u) acc[u] = cmul_add(m, x[u][c], acc[u]);
        }
        uint32_t roff = 0;
#pragma unroll
        for (int b = 0; b < K; ++b)
          if ((r >> b) & 1) roff += lo[b] + 1;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (g0 + u * kTThreads < ng) {
            const uint32_t o = base[u] + roff;
            sv[o] = acc[u];
            if (stats) {
              const double p = (double)acc[u].x * acc[u].x + (double)acc[u].y * acc[u].y;
              lt += p;
              ld += p * S.stab[__popc(o & smask)];
            }
          }
        }
      }
    }
    t += lt;
    d += ld;
  }

  static __device__ void dispatch_gate(float2 *sv, uint32_t n, const TOp &op, const float2 *M, Shared &S,
                                double &t, double &d) {
    if (S.pend) {
      switch (op.k) {
      case 1: gate_pass<1, true>(sv, n, op, M, S, t, d); break;
      case 2: gate_pass<2, true>(sv, n, op, M, S, t, d); break;
      case 3: gate_pass<3, true>(sv, n, op, M, S, t, d); break;
      default: gate_pass<4, true>(sv, n, op, M, S, t, d); break;
      }
    } else {
      switch (op.k) {
      case 1: gate_pass<1, false>(sv, n, op, M, S, t, d); break;
      case 2: gate_pass<2, false>(sv, n, op, M, S, t, d); break;
      case 3: gate_pass<3, false>(sv, n, op, M, S, t, d); break;
      default: gate_pass<4, false>(sv, n, op, M, S, t, d); break;
      }
    }
  }

  // Stage a 2^k x 2^k matrix into shared memory.
  static __device__ void stage_matrix(float2 *Msm, const float2 *pool, uint32_t off, uint32_t entries) {
    for (uint32_t i = threadIdx.x; i < entries; i += kTThreads) Msm[i] = pool[off + i];
    __syncthreads();
  }

  // Materialise the pending diagonal (and optionally compute sums):
  // t = sum |a|^2, d = sum |a|^2 * w(i) with w = (1-g)^popc(i & mask), j = g * sum_{bit q} |a|^2.
  static __device__ __noinline__ void stats_pass(float2 *sv, uint32_t n, Shared &S, uint32_t mask, double g, uint32_t q,
                             double &t, double &d, double &j) {
    t = d = j = 0;
    fill_stab(S, g);
    const uint32_t N = 1u << n;
    for (uint32_t i = threadIdx.x; i < N; i += kTThreads) {
      float2 v = sv[i];
      if (S.pend) {
        const float f = S.dtab[__popc(i & S.pmask)];
        v.x *= f;
        v.y *= f;
        sv[i] = v;
      }
      const double p = (double)v.x * v.x + (double)v.y * v.y;
      t += p;
      d += p * S.stab[__popc(i & mask)];
      if ((i >> q) & 1) j += p;
    }
    __syncthreads();
    if (threadIdx.x == 0) S.pend = 0;
    block_sum3(S, t, d, j);
    j *= g;
  }

  static __device__ void set_pending(Shared &S, uint32_t mask, double gamma, double scale) {
    if (threadIdx.x == 0) {
      S.pend = 1;
      S.pmask = mask;
      const double s = sqrt(1.0 - gamma);
      double f = scale;
      for (uint32_t c = 0; c <= kTrajMaxQubits; ++c) {
        S.dtab[c] = (float)f;
        f *= s;
      }
    }
    __syncthreads();
  }

  // Elementwise single-qubit damping branch on qubit q: jump -> x0 = sqrt(g) x1, x1 = 0;
  // no jump -> x1 *= sqrt(1 - g).
  static __device__ __noinline__ void damp_apply(float2 *sv, uint32_t n, uint32_t q, double g, bool jump) {
    const uint32_t npair = 1u << (n - 1);
    const uint32_t lo = (1u << q) - 1;
    const float sj = (float)sqrt(g), sn = (float)sqrt(1.0 - g);
    for (uint32_t p = threadIdx.x; p < npair; p += kTThreads) {
      const uint32_t i0 = ((p & ~lo) << 1) | (p & lo), i1 = i0 | (1u << q);
      const float2 x1 = sv[i1];
      if (jump) {
        sv[i0] = make_float2(sj * x1.x, sj * x1.y);
        sv[i1] = make_float2(0.f, 0.f);
      } else {
        sv[i1] = make_float2(sn * x1.x, sn * x1.y);
      }
    }
    __syncthreads();
  }

  // General single-qubit channel: p_j = ||K_j psi||^2 (FP64), pick j, apply K_j / sqrt(p_j).
  static __device__ __noinline__ void chan_op(float2 *sv, uint32_t n, const TOp &op, const float2 *pool,
                                       float2 *Msm, Shared &S, uint64_t seed, uint32_t traj,
                                       uint32_t &ev) {
    const uint32_t N = 1u << n;
    stage_matrix(Msm, pool, op.mat, 4 * op.nk);
    const uint32_t q = op.q[0];
    const uint32_t lo = (1u << q) - 1;
    double pj[4] = {0, 0, 0, 0};
    for (uint32_t p = threadIdx.x; p < N / 2; p += kTThreads) {
      const uint32_t i0 = ((p & ~lo) << 1) | (p & lo), i1 = i0 | (1u << q);
      const float2 x0 = pend_load(sv, i0, S), x1 = pend_load(sv, i1, S);
      for (uint32_t b = 0; b < op.nk; ++b) {
        const float2 y0 = cmul_add(Msm[4 * b + 1], x1, cmul_add(Msm[4 * b], x0, make_float2(0, 0)));
        const float2 y1 = cmul_add(Msm[4 * b + 3], x1, cmul_add(Msm[4 * b + 2], x0, make_float2(0, 0)));
        pj[b] += (double)y0.x * y0.x + (double)y0.y * y0.y + (double)y1.x * y1.x + (double)y1.y * y1.y;
      }
    }
    double a = pj[0], b = pj[1], c = pj[2];
    block_sum3(S, a, b, c);
    double d3 = pj[3], z0 = 0, z1 = 0;
    block_sum3(S, d3, z0, z1);
    const double tot[4] = {a, b, c, d3};
    double sum = 0;
    for (uint32_t bb = 0; bb < op.nk; ++bb) sum += tot[bb];
    const double v = philox_uniform(seed, traj, ev++) * sum;
    uint32_t pick = op.nk - 1;
    double acc = 0;
    for (uint32_t bb = 0; bb < op.nk; ++bb) {
      acc += tot[bb];
      if (v < acc) {
        pick = bb;
        break;
      }
    }
    const float sc = (float)(tot[pick] > 0 ? 1.0 / sqrt(tot[pick]) : 0.0);
    const float2 *K = Msm + 4 * pick;
    for (uint32_t p = threadIdx.x; p < N / 2; p += kTThreads) {
      const uint32_t i0 = ((p & ~lo) << 1) | (p & lo), i1 = i0 | (1u << q);
      const float2 x0 = pend_load(sv, i0, S), x1 = pend_load(sv, i1, S);
      const float2 y0 = cmul_add(K[1], x1, cmul_add(K[0], x0, make_float2(0, 0)));
      const float2 y1 = cmul_add(K[3], x1, cmul_add(K[2], x0, make_float2(0, 0)));
      sv[i0] = make_float2(y0.x * sc, y0.y * sc);
      sv[i1] = make_float2(y1.x * sc, y1.y * sc);
    }
    __syncthreads();
    if (threadIdx.x == 0) S.pend = 0;
    __syncthreads();
  }

  // Applies a Pauli error op (one of three k-qubit matrices) as a gate pass.
  static __device__ __noinline__ void err_apply(float2 *sv, uint32_t n, const TOp &op, double u,
                                         const float2 *pool, float2 *Msm, Shared &S) {
    const uint32_t which = min(2u, (uint32_t)(u / (double)op.prob * 3.0));
    const uint32_t e = 1u << (2 * op.k);
    stage_matrix(Msm, pool, op.mat + which * e, e);
    TOp g = op;
    g.stats = 0;
    double t = 0, d = 0;
    dispatch_gate(sv, n, g, Msm, S, t, d);
    __syncthreads();
    if (threadIdx.x == 0) S.pend = 0;
    __syncthreads();
  }

  // Amplitude damping on op.mask: exact sampling of the joint jump pattern.
  static __device__ __noinline__ void damp_op(float2 *sv, uint32_t n, const TOp &op, Shared &S,
                                       uint64_t seed, uint32_t traj, uint32_t &ev, double T,
                                       double Dd, bool stats_valid) {
    const double g = (double)op.gamma;
    if (!stats_valid) {
      double j;
      stats_pass(sv, n, S, op.mask, g, 0, T, Dd, j);
    }
    const double u = philox_uniform(seed, traj, ev++);
    if (u * T < Dd) {  // no jump on any qubit of the mask
      set_pending(S, op.mask, g, 1.0 / sqrt(Dd));
      return;
    }
    // at least one jump: sample qubit by qubit, conditioned on a jump occurring
    if (S.pend) {
      double a, b, c;
      stats_pass(sv, n, S, 0, 0.0, 0, a, b, c);
    }
    bool need = true;
    for (uint32_t q = 0; q < n; ++q) {
      if (!((op.mask >> q) & 1)) continue;
      const uint32_t rem = op.mask & ~((1u << q) - 1);
      double t, zsum, j;
      stats_pass(sv, n, S, rem, g, q, t, zsum, j);
      const double p1 = need ? (t - zsum > 0 ? j / (t - zsum) : 1.0) : (t > 0 ? j / t : 0.0);
      const double v = philox_uniform(seed, traj, ev++);
      const bool jump = v < p1;
      damp_apply(sv, n, q, g, jump);
      if (jump) need = false;
    }
    double t, a, b;
    stats_pass(sv, n, S, 0, 0.0, 0, t, a, b);
    set_pending(S, 0, 0.0, t > 0 ? 1.0 / sqrt(t) : 1.0);
  }

  // End of a trajectory: <Z_q> for every qubit and one sampled bitstring.
  static __device__ __noinline__ void finish(float2 *sv, uint32_t n, Shared &S, double *csum, uint64_t seed,
                                      uint32_t traj, double *z_row, uint32_t *sample_slot) {
    {
      double t, a, b;
      stats_pass(sv, n, S, 0, 0.0, 0, t, a, b);  // materialise the pending diagonal
    }
    const uint32_t N = 1u << n;
    const uint32_t c = n > kTLogThreads ? n - kTLogThreads : 0;  // bits inside a thread's chunk
    const uint32_t chunk = 1u << c;
    const bool active = (threadIdx.x << c) < N;
    const uint32_t base = threadIdx.x << c;
    double my = 0;
    if (active)
      for (uint32_t i = 0; i < chunk; ++i) {
        const float2 v = sv[base + i];
        my += (double)v.x * v.x + (double)v.y * v.y;
      }
    csum[threadIdx.x] = my;
    __syncthreads();
    // qubits inside a chunk, three per block reduction
    for (uint32_t q0 = 0; q0 < c; q0 += 3) {
      double acc[3] = {0, 0, 0};
      if (active)
        for (uint32_t i = 0; i < chunk; ++i) {
          const float2 v = sv[base + i];
          const double p = (double)v.x * v.x + (double)v.y * v.y;
          for (uint32_t j = 0; j < 3; ++j)
            if (q0 + j < c && ((i >> (q0 + j)) & 1)) acc[j] += p;
        }
      block_sum3(S, acc[0], acc[1], acc[2]);
      if (threadIdx.x < 3 && q0 + threadIdx.x < c) z_row[q0 + threadIdx.x] = acc[threadIdx.x];
    }
    // qubits that index the threads: thread j sums the chunk sums with bit j set
    const uint32_t nthr = N >> c;
    if (threadIdx.x < n - c) {
      double x = 0;
      for (uint32_t tt = 0; tt < nthr; ++tt)
        if ((tt >> threadIdx.x) & 1) x += csum[tt];
      z_row[c + threadIdx.x] = x;
    }
    if (threadIdx.x == 0) {
      double tot = 0;
      for (uint32_t tt = 0; tt < nthr; ++tt) tot += csum[tt];
      S.vals[3] = tot;
      // inverse-CDF sample: find the chunk, then the amplitude (a target that
      // rounding leaves past the end takes the last one of nonzero weight)
      const double target = philox_uniform(seed, traj, 0xFFFFFFF0u) * tot;
      double acc = 0, acc_t = 0;
      uint32_t tsel = nthr;
      for (uint32_t tt = 0; tt < nthr; ++tt) {
        if (csum[tt] > 0) {
          tsel = tt;
          acc_t = acc;
        }
        if (acc + csum[tt] > target) break;
        acc += csum[tt];
      }
      acc = acc_t;
      if (tsel == nthr) tsel = 0;  // an all-zero state (cannot arise from normalised branches)
      uint32_t isel = tsel << c;
      for (uint32_t i = 0; i < chunk; ++i) {
        const float2 v = sv[(tsel << c) + i];
        const double p = (double)v.x * v.x + (double)v.y * v.y;
        if (p > 0) isel = (tsel << c) + i;
        acc += p;
        if (acc > target) break;
      }
      if (sample_slot) *sample_slot = isel;
    }
    __syncthreads();
    const double tot = S.vals[3];
    if (threadIdx.x < n) {
      const double p1 = z_row[threadIdx.x];
      z_row[threadIdx.x] = tot > 0 ? 1.0 - 2.0 * p1 / tot : 0.0;
    }
    __syncthreads();
  }
};

template <int NT>
__global__ void __launch_bounds__(NT, 1)
    k_trajectories(const TOp *__restrict__ ops, uint32_t n_ops, const float2 *__restrict__ pool,
                   float2 *__restrict__ ws, uint32_t n, const TRun *__restrict__ run,
                   double *__restrict__ out_z, uint32_t *__restrict__ out_sample) {
  __shared__ Shared S;
  __shared__ float2 Msm[1 << (2 * kTrajMaxGate)];
  __shared__ double csum[NT];
  using Tr = Traj<NT>;
  const uint32_t n_traj = run->n_traj;
  const uint64_t seed = run->seed;
  const uint32_t N = 1u << n;
  float2 *sv = ws + ((size_t)blockIdx.x << n);
  for (uint32_t lt = blockIdx.x; lt < n_traj; lt += gridDim.x) {
    const uint32_t traj = run->first + lt;  // draws depend on the global index only
    for (uint32_t i = threadIdx.x; i < N; i += NT)
      sv[i] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
    if (threadIdx.x == 0) S.pend = 0;
    __syncthreads();
    uint32_t ev = 0;
    bool stats_valid = false;
    double T = 1.0, Dd = 1.0;
    for (uint32_t oi = 0; oi < n_ops; ++oi) {
      const TOp op = ops[oi];
      if (op.type == T_GATE) {
        if (op.stats) Tr::fill_stab(S, (double)op.sgamma);
        Tr::stage_matrix(Msm, pool, op.mat, 1u << (2 * op.k));
        double t = 0, d = 0, z = 0;
        Tr::dispatch_gate(sv, n, op, Msm, S, t, d);
        __syncthreads();
        if (threadIdx.x == 0) S.pend = 0;
        if (op.stats) {
          Tr::block_sum3(S, t, d, z);
          T = t;
          Dd = d;
        } else {
          __syncthreads();
        }
        stats_valid = op.stats != 0;
        if (op.nerr) {
          // all error sites of this block decide in parallel (event ev + e for site e)
          int fired = 0;
          if (threadIdx.x < op.nerr)
            fired = philox_uniform(seed, traj, ev + threadIdx.x) < (double)ops[oi + 1 + threadIdx.x].prob;
          if (__syncthreads_or(fired)) {
            for (uint32_t e = 0; e < op.nerr; ++e) {
              const TOp eo = ops[oi + 1 + e];
              const double u = philox_uniform(seed, traj, ev + e);
              if (u < (double)eo.prob) {
                Tr::err_apply(sv, n, eo, u, pool, Msm, S);
                stats_valid = false;
              }
            }
          }
          ev += op.nerr;
          oi += op.nerr;
        }
      } else if (op.type == T_ERR) {  // not preceded by a gate block (kept for completeness)
        const double u = philox_uniform(seed, traj, ev++);
        if (u < (double)op.prob) {
          Tr::err_apply(sv, n, op, u, pool, Msm, S);
          stats_valid = false;
        }
      } else if (op.type == T_DAMP) {
        Tr::damp_op(sv, n, op, S, seed, traj, ev, T, Dd, stats_valid);
        stats_valid = false;
      } else if (op.type == T_CHAN) {
        Tr::chan_op(sv, n, op, pool, Msm, S, seed, traj, ev);
        stats_valid = false;
      }
    }
    Tr::finish(sv, n, S, csum, seed, traj, out_z + (size_t)lt * n, out_sample ? out_sample + lt : nullptr);
  }
}

constexpr uint32_t kTrajMagic = 0xCB2077A1u;

// Threads per CTA when the program does not fix them: 1024 for states of 15 to
// 17 qubits (slices larger than L1 but held in L2, so passes are bound by loads
// in flight), 512 otherwise (issue-bound gate arithmetic).
unsigned auto_threads(uint32_t n) { return n >= 15 && n <= 17 ? 1024u : 512u; }

// Trajectories in flight when the program does not fix them: one per SM, unless
// the slices of one per SM overflow L2 while those of at least half as many
// still fit in 89% of it (17 qubits: 112 CTAs x 1 MB instead of 148, 1.8x the
// throughput); beyond that the passes stream from HBM either way.
unsigned auto_ctas(uint32_t n) {
  const unsigned sms = (unsigned)cb2::sm_count();
  int dev = 0, l2 = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess || l2 <= 0) {
    cudaGetLastError();
    return sms;
  }
  const uint64_t slice = sizeof(float2) << n;
  const uint64_t fit = (uint64_t)l2 * 89 / 100 / slice;
  return fit >= sms || fit < sms / 2 ? sms : (unsigned)fit;
}

// No access-policy window: a persisting-L2 set-aside sized for the workspace
// gave the trajectories 4% at 16 qubits but, being a limit of the whole
// context, cut every later streaming gate pass of the process from 6.3 to
// 2.8 TB/s until it was set back to 0.
cudaError_t launch_trajectories(unsigned grid, unsigned threads, cudaStream_t s, const TOp *ops,
                                uint32_t n_ops, const float2 *pool, float2 *ws, uint32_t n,
                                const TRun *run, double *z, uint32_t *sample) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  if (threads == 1024)
    return cudaLaunchKernelEx(&cfg, k_trajectories<1024>, ops, n_ops, pool, ws, n, run, z, sample);
  return cudaLaunchKernelEx(&cfg, k_trajectories<512>, ops, n_ops, pool, ws, n, run, z, sample);
}

// Device buffers of trajectory programs come from a process-wide cache keyed by
// (device, exact size).  cudaFree synchronises the whole device, and a serving
// loop creates and drops one program per noisy request while other requests
// run on other streams.  A dropped program's buffers are idle (cast_b200_traj_run
// returns only after its work completes), so they wait here for reuse, up to
// 8 GiB in all; beyond that they are freed.  The device of a returned buffer is
// read from the pointer itself, so a process that switches devices with
// cast_b200_set_device never receives another device's memory.
std::mutex g_buf_mu;
std::multimap<std::pair<int, size_t>, void *> g_buf_cache;
size_t g_buf_cached = 0;
constexpr size_t kBufCacheMax = 8ull << 30;

cudaError_t buf_alloc(void **p, size_t bytes) {
  int dev = 0;
  const cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess) return rc;
  {
    std::lock_guard<std::mutex> lock(g_buf_mu);
    auto it = g_buf_cache.find({dev, bytes});
    if (it != g_buf_cache.end()) {
      *p = it->second;
      g_buf_cache.erase(it);
      g_buf_cached -= bytes;
      return cudaSuccess;
    }
  }
  return cudaMalloc(p, bytes);
}

void buf_free(void *p, size_t bytes) {
  if (!p) return;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeDevice) {
    std::lock_guard<std::mutex> lock(g_buf_mu);
    if (g_buf_cached + bytes <= kBufCacheMax) {
      g_buf_cache.emplace(std::make_pair(attr.device, bytes), p);
      g_buf_cached += bytes;
      return;
    }
  }
  cudaFree(p);
}

struct TrajProgram {
  uint32_t magic = kTrajMagic;
  uint32_t n = 0;
  std::vector<TOp> ops;
  std::vector<float2> pool;
  bool dirty = true;
  TOp *d_ops = nullptr;
  float2 *d_pool = nullptr;
  float2 *d_ws = nullptr;
  size_t ws_ctas = 0;
  size_t ops_bytes = 0, pool_bytes = 0, ws_bytes = 0, z_bytes = 0, sample_bytes = 0;
  TRun *d_run = nullptr;
  double *d_z = nullptr;
  uint32_t *d_sample = nullptr;
  size_t out_cap = 0;
  cudaGraphExec_t graph = nullptr;
  void *graph_stream = nullptr;
  unsigned graph_grid = 0;
  unsigned threads = 0;  // threads per CTA: 512, 1024, or 0 for auto_threads(n)
  unsigned max_ctas = 0; // CTAs (trajectories in flight), or 0 for auto_ctas(n)
  unsigned graph_threads = 0;
  std::mutex mu;

  ~TrajProgram() {
    if (graph) cudaGraphExecDestroy(graph);
    buf_free(d_ops, ops_bytes);
    buf_free(d_pool, pool_bytes);
    buf_free(d_ws, ws_bytes);
    buf_free(d_run, sizeof(TRun));
    buf_free(d_z, z_bytes);
    buf_free(d_sample, sample_bytes);
  }

  uint32_t push_matrix(const cast_complex64_t *m, size_t entries) {
    const uint32_t off = (uint32_t)pool.size();
    for (size_t i = 0; i < entries; ++i) pool.push_back(make_float2((float)m[i].re, (float)m[i].im));
    return off;
  }

  void mark_stats() {
    for (auto &o : ops) o.stats = o.nerr = 0;
    for (size_t i = 0; i < ops.size(); ++i) {
      if (ops[i].type != T_GATE) continue;
      uint32_t e = 0;
      while (i + 1 + e < ops.size() && ops[i + 1 + e].type == T_ERR && e < (uint32_t)kTMinThreads) ++e;
      ops[i].nerr = e;
    }
    for (size_t i = 0; i < ops.size(); ++i) {
      if (ops[i].type != T_DAMP) continue;
      size_t j = i;
      while (j > 0 && ops[j - 1].type == T_ERR) --j;
      if (j > 0 && ops[j - 1].type == T_GATE) {
        ops[j - 1].stats = 1;
        ops[j - 1].smask = ops[i].mask;
        ops[j - 1].sgamma = ops[i].gamma;
      }
    }
  }

  bool upload(std::string &err) {
    if (!dirty) return true;
    mark_stats();
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    buf_free(d_ops, ops_bytes);
    buf_free(d_pool, pool_bytes);
    d_ops = nullptr;
    d_pool = nullptr;
    ops_bytes = pool_bytes = 0;
    const size_t ob = sizeof(TOp) * std::max<size_t>(1, ops.size());
    const size_t pb = sizeof(float2) * std::max<size_t>(1, pool.size());
    if (!cuda_ok(buf_alloc(reinterpret_cast<void **>(&d_ops), ob), "cudaMalloc (trajectory ops)", err))
      return false;
    ops_bytes = ob;
    if (!cuda_ok(buf_alloc(reinterpret_cast<void **>(&d_pool), pb), "cudaMalloc (trajectory matrices)", err))
      return false;
    pool_bytes = pb;
    if (!ops.empty() &&
        !cuda_ok(cudaMemcpy(d_ops, ops.data(), sizeof(TOp) * ops.size(), cudaMemcpyHostToDevice),
                 "cudaMemcpy (trajectory ops)", err))
      return false;
    if (!pool.empty() &&
        !cuda_ok(cudaMemcpy(d_pool, pool.data(), sizeof(float2) * pool.size(),
                            cudaMemcpyHostToDevice),
                 "cudaMemcpy (trajectory matrices)", err))
      return false;
    dirty = false;
    return true;
  }
};

TrajProgram *as_traj(void *p) {
  TrajProgram *t = static_cast<TrajProgram *>(p);
  return t && t->magic == kTrajMagic ? t : nullptr;
}

bool check_qubits(const TrajProgram &p, const uint32_t *q, uint32_t k, std::string &err) {
  if (!q || k == 0 || k > kTrajMaxGate) {
    err = "trajectory gates act on 1.." + std::to_string(kTrajMaxGate) + " qubits";
    return false;
  }
  for (uint32_t b = 0; b < k; ++b) {
    if (q[b] >= p.n) {
      err = "qubit out of range";
      return false;
    }
    if (b && q[b - 1] >= q[b]) {
      err = "qubits must be distinct and ascending";
      return false;
    }
  }
  return true;
}

}  // namespace

extern "C" {

void *cast_b200_traj_create(uint32_t n_qubits, char *err_buf, size_t err_buf_len) {
  if (n_qubits == 0 || n_qubits > kTrajMaxQubits) {
    cb2::write_err(err_buf, err_buf_len,
                   "trajectory statevectors support 1.." + std::to_string(kTrajMaxQubits) + " qubits");
    return nullptr;
  }
  try {
    TrajProgram *p = new TrajProgram;
    p->n = n_qubits;
    cb2::clear_err(err_buf, err_buf_len);
    return p;
  } catch (const std::exception &e) {
    cb2::write_err(err_buf, err_buf_len, e.what());
    return nullptr;
  }
}

void cast_b200_traj_destroy(void *prog) {
  TrajProgram *p = as_traj(prog);
  if (!p) return;
  p->magic = 0;
  delete p;
}

int cast_b200_traj_add_gate(void *prog, const cast_complex64_t *matrix, const uint32_t *qubits,
                            uint32_t k, char *err_buf, size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  std::string err;
  if (!p || !matrix) err = "invalid trajectory program or matrix";
  else if (check_qubits(*p, qubits, k, err)) {
    std::lock_guard<std::mutex> lock(p->mu);
    TOp o{};
    o.type = T_GATE;
    o.k = k;
    for (uint32_t b = 0; b < k; ++b) o.q[b] = qubits[b];
    o.mat = p->push_matrix(matrix, 1ull << (2 * k));
    p->ops.push_back(o);
    p->dirty = true;
    cb2::clear_err(err_buf, err_buf_len);
    return 0;
  }
  cb2::write_err(err_buf, err_buf_len, err);
  return 1;
}

int cast_b200_traj_add_pauli_error(void *prog, double prob, const cast_complex64_t *mats,
                                   char *err_buf, size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  if (!p || !mats || prob < 0.0 || prob > 1.0) {
    cb2::write_err(err_buf, err_buf_len, "invalid trajectory program, matrices or probability");
    return 1;
  }
  std::lock_guard<std::mutex> lock(p->mu);
  if (p->ops.empty() || (p->ops.back().type != T_GATE && p->ops.back().type != T_ERR)) {
    cb2::write_err(err_buf, err_buf_len, "a Pauli error must follow the gate block it belongs to");
    return 1;
  }
  size_t gi = p->ops.size() - 1;
  while (p->ops[gi].type != T_GATE) --gi;
  TOp o = p->ops[gi];
  o.type = T_ERR;
  o.prob = (float)prob;
  o.mat = p->push_matrix(mats, 3ull << (2 * o.k));
  p->ops.push_back(o);
  p->dirty = true;
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_traj_add_damping(void *prog, uint32_t mask, double gamma, char *err_buf,
                               size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  if (!p || gamma < 0.0 || gamma >= 1.0 || mask == 0 || (p->n < 32 && (mask >> p->n) != 0)) {
    cb2::write_err(err_buf, err_buf_len, "invalid damping mask or rate");
    return 1;
  }
  std::lock_guard<std::mutex> lock(p->mu);
  TOp o{};
  o.type = T_DAMP;
  o.mask = mask;
  o.gamma = (float)gamma;
  p->ops.push_back(o);
  p->dirty = true;
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_traj_add_channel(void *prog, uint32_t qubit, const cast_complex64_t *kraus,
                               uint32_t n_kraus, char *err_buf, size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  if (!p || !kraus || n_kraus == 0 || n_kraus > 4 || qubit >= p->n) {
    cb2::write_err(err_buf, err_buf_len, "invalid channel (1..4 Kraus operators on one qubit)");
    return 1;
  }
  std::lock_guard<std::mutex> lock(p->mu);
  TOp o{};
  o.type = T_CHAN;
  o.k = 1;
  o.q[0] = qubit;
  o.nk = n_kraus;
  o.mat = p->push_matrix(kraus, 4ull * n_kraus);
  p->ops.push_back(o);
  p->dirty = true;
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_traj_set_launch(void *prog, uint32_t threads, uint32_t max_ctas, char *err_buf,
                              size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  if (!p || (threads != 0 && threads != 512 && threads != 1024)) {
    cb2::write_err(err_buf, err_buf_len, "threads per CTA must be 512, 1024 or 0 (by state size)");
    return 1;
  }
  std::lock_guard<std::mutex> lock(p->mu);
  p->threads = threads;
  p->max_ctas = max_ctas;
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

uint32_t cast_b200_traj_num_qubits(const void *prog) {
  const TrajProgram *p = static_cast<const TrajProgram *>(prog);
  return p && p->magic == kTrajMagic ? p->n : 0;
}

int cast_b200_traj_get_op(const void *prog, uint32_t index, uint32_t *out_type, uint32_t *out_k,
                          uint32_t *out_qubits, double *out_prob, uint32_t *out_mask,
                          uint32_t *out_n_mats, cast_complex64_t *out_mats, size_t out_mats_len) {
  const TrajProgram *p = static_cast<const TrajProgram *>(prog);
  if (!p || p->magic != kTrajMagic || index >= p->ops.size()) return 1;
  const TOp &o = p->ops[index];
  size_t entries = 0;
  uint32_t nm = 0;
  double prob = 0;
  switch (o.type) {
  case T_GATE: nm = 1; entries = 1ull << (2 * o.k); break;
  case T_ERR: nm = 3; entries = 3ull << (2 * o.k); prob = o.prob; break;
  case T_DAMP: prob = o.gamma; break;
  default: nm = o.nk; entries = 4ull * o.nk; break;
  }
  if (out_type) *out_type = o.type;
  if (out_k) *out_k = o.k;
  if (out_qubits)
    for (uint32_t b = 0; b < o.k && b < kTrajMaxGate; ++b) out_qubits[b] = o.q[b];
  if (out_prob) *out_prob = prob;
  if (out_mask) *out_mask = o.mask;
  if (out_n_mats) *out_n_mats = nm;
  if (out_mats) {
    if (out_mats_len < entries) return 1;
    for (size_t e = 0; e < entries; ++e)
      out_mats[e] = {p->pool[o.mat + e].x, p->pool[o.mat + e].y};
  }
  return 0;
}

uint32_t cast_b200_traj_num_ops(const void *prog) {
  const TrajProgram *p = static_cast<const TrajProgram *>(prog);
  return p && p->magic == kTrajMagic ? (uint32_t)p->ops.size() : 0;
}

int cast_b200_traj_run(void *prog, uint32_t n_traj, uint64_t seed, double *out_z,
                       uint32_t *out_samples, void *stream, int use_graph, char *err_buf,
                       size_t err_buf_len) {
  return cast_b200_traj_run_range(prog, 0, n_traj, seed, out_z, out_samples, stream, use_graph,
                                  err_buf, err_buf_len);
}

int cast_b200_traj_run_range(void *prog, uint32_t first, uint32_t n_traj, uint64_t seed,
                             double *out_z, uint32_t *out_samples, void *stream, int use_graph,
                             char *err_buf, size_t err_buf_len) {
  TrajProgram *p = as_traj(prog);
  if (p && (uint64_t)first + n_traj > 0xFFFFFFFFull) {
    cb2::write_err(err_buf, err_buf_len, "trajectory range exceeds 2^32 indices");
    return 1;
  }
  if (!p || !out_z || n_traj == 0) {
    cb2::write_err(err_buf, err_buf_len, "invalid trajectory program, output or count");
    return 1;
  }
  try {
    std::lock_guard<std::mutex> lock(p->mu);
    std::string err;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!p->upload(err)) {
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
    const unsigned ctas = p->max_ctas ? p->max_ctas : auto_ctas(p->n);
    const unsigned grid = (unsigned)std::min<uint64_t>(n_traj, ctas);
    const unsigned threads = p->threads ? p->threads : auto_threads(p->n);
    if (p->ws_ctas < grid) {
      buf_free(p->d_ws, p->ws_bytes);
      p->d_ws = nullptr;
      p->ws_bytes = 0;
      if (!cuda_ok(buf_alloc(reinterpret_cast<void **>(&p->d_ws), (sizeof(float2) << p->n) * grid),
                   "cudaMalloc (trajectory workspace)", err)) {
        cb2::write_err(err_buf, err_buf_len, err);
        return 1;
      }
      p->ws_ctas = grid;
      p->ws_bytes = (sizeof(float2) << p->n) * grid;
      if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
      }
    }
    if (!p->d_run &&
        !cuda_ok(buf_alloc(reinterpret_cast<void **>(&p->d_run), sizeof(TRun)), "cudaMalloc (run)", err)) {
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
    if (p->out_cap < n_traj) {
      buf_free(p->d_z, p->z_bytes);
      buf_free(p->d_sample, p->sample_bytes);
      p->d_z = nullptr;
      p->d_sample = nullptr;
      p->z_bytes = p->sample_bytes = 0;
      if (!cuda_ok(buf_alloc(reinterpret_cast<void **>(&p->d_z), sizeof(double) * n_traj * p->n),
                   "cudaMalloc (z)", err)) {
        cb2::write_err(err_buf, err_buf_len, err);
        return 1;
      }
      p->z_bytes = sizeof(double) * n_traj * p->n;
      if (!cuda_ok(buf_alloc(reinterpret_cast<void **>(&p->d_sample), sizeof(uint32_t) * n_traj),
                   "cudaMalloc (samples)", err)) {
        cb2::write_err(err_buf, err_buf_len, err);
        return 1;
      }
      p->sample_bytes = sizeof(uint32_t) * n_traj;
      p->out_cap = n_traj;
      if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
      }
    }
    TRun r{n_traj, first, seed};
    if (!cuda_ok(cudaMemcpyAsync(p->d_run, &r, sizeof(r), cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync (run parameters)", err)) {
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
    const uint32_t n_ops = (uint32_t)p->ops.size();
    if (use_graph && s) {
      if (p->graph && (p->graph_stream != stream || p->graph_grid != grid || p->graph_threads != threads)) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
      }
      if (!p->graph) {
        cudaGraph_t gph = nullptr;
        if (!cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal),
                     "cudaStreamBeginCapture", err)) {
          cb2::write_err(err_buf, err_buf_len, err);
          return 1;
        }
        const cudaError_t lrc = launch_trajectories(grid, threads, s, p->d_ops, n_ops, p->d_pool,
                                                    p->d_ws, p->n, p->d_run, p->d_z, p->d_sample);
        const cudaError_t erc = cudaStreamEndCapture(s, &gph);
        if (!cuda_ok(lrc, "trajectory kernel capture", err) ||
            !cuda_ok(erc, "cudaStreamEndCapture", err) ||
            !cuda_ok(cudaGraphInstantiate(&p->graph, gph, 0), "cudaGraphInstantiate", err)) {
          if (gph) cudaGraphDestroy(gph);
          cb2::write_err(err_buf, err_buf_len, err);
          return 1;
        }
        cudaGraphDestroy(gph);
        p->graph_stream = stream;
        p->graph_grid = grid;
        p->graph_threads = threads;
      }
      if (!cuda_ok(cudaGraphLaunch(p->graph, s), "cudaGraphLaunch", err)) {
        cb2::write_err(err_buf, err_buf_len, err);
        return 1;
      }
    } else {
      if (!cuda_ok(launch_trajectories(grid, threads, s, p->d_ops, n_ops, p->d_pool, p->d_ws, p->n,
                                       p->d_run, p->d_z, p->d_sample),
                   "trajectory kernel launch", err)) {
        cb2::write_err(err_buf, err_buf_len, err);
        return 1;
      }
    }
    if (!cuda_ok(cudaMemcpyAsync(out_z, p->d_z, sizeof(double) * n_traj * p->n,
                                 cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (z)", err) ||
        (out_samples &&
         !cuda_ok(cudaMemcpyAsync(out_samples, p->d_sample, sizeof(uint32_t) * n_traj,
                                  cudaMemcpyDeviceToHost, s),
                  "cudaMemcpyAsync (samples)", err)) ||
        !cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (trajectories)", err)) {
      // The kernel may already be queued: let it finish before returning, so
      // that no buffer of this program is handed on (buffer cache) in use.
      cudaStreamSynchronize(s);
      cb2::write_err(err_buf, err_buf_len, err);
      return 1;
    }
    cb2::clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &e) {
    cb2::write_err(err_buf, err_buf_len, e.what());
    return 1;
  }
}

}  // extern "C"
