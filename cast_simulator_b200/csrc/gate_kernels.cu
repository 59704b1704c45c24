// Gate-application kernels for sm_100a: apply a fused k-qubit complex gate
// (2^k x 2^k, row-major) in place to an interleaved re/im statevector of 2^n
// amplitudes, in FP32 or FP64.
//
// This is the hot path the reference generates per gate with LLVM NVPTX
// (src/cpp/cuda/cuda_gen.cpp:174-342: combo -> base offset by bit insertion,
// 2^k loads, straight-line matvec, 2^k stores, persistent grid-stride loop).
// Here the kernels are precompiled templates on (scalar type, k) and the
// matrix is data:
//
//  * k <= 5 ("register" kernels): one thread owns one gather group of 2^k
//    amplitudes in registers.  The matrix travels in the kernel parameter
//    block, so every matrix scalar is a constant-bank operand of the FMA that
//    uses it (no load instruction, uniform across the warp) - the data-side
//    equivalent of the reference's baked-in immediates.  Consecutive threads
//    take consecutive groups, i.e. they walk the lowest non-target qubits, so
//    each of the 2^k 128-bit (f64) / 64-bit (f32) loads of a warp is one
//    contiguous run whenever the lowest target is >= 5 and stays within the
//    same cache lines across the 2^k loads otherwise.
//  * k = 6, 7 ("staged" kernels): a CTA copies a tile of 32..128 groups into
//    shared memory with asynchronous coalesced copies, then computes the
//    2^k x 2^k by 2^k x G complex product register-tiled (each thread a block
//    of rows x groups) and stores straight back to HBM.  These are bound by the
//    FP32 / FP64 FMA pipes, not HBM.
//
// Zero / +-1 matrix scalars (classified on the host with the reference's
// tolerances) are exact, so dense evaluation reproduces the reference's
// skipped / sign-flipped products bit for bit up to summation order.
#include "internal.hpp"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cuda_pipeline.h>

namespace cb2 {

namespace {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Target qubits (ascending) with their low-bit masks, passed by value.
struct Targets {
  uint64_t lo_mask[kMaxGateQubits];  // (1 << q_b) - 1
  uint64_t stride[kMaxGateQubits];   // 1 << q_b (amplitude units)
};

// 4-qubit gates use three real products per complex multiply-add (the 3M
// method, Higham, "Accuracy and Stability of Numerical Algorithms", 2nd ed.,
// sec. 23.2.4): for M = c + i d and x = a + i b,
//   S1 += c (a + b),  S2 += a (d - c),  S3 += b (c + d),
//   Re(Mx) = S1 - S3,  Im(Mx) = S1 + S2,
// with a + b formed once per amplitude and c, d - c, c + d formed on the host.
// That is 48 FMAs and 3 adds per row against 64 FMAs.  At k = 4 the FP64 pass
// is FMA-bound at the power-capped SM clock (about 1.35 GHz); the rounding
// error stays within a small multiple of the 4-product form's (Higham,
// Lemma 3.7 and sec. 23.2.4), and an exact zero entry still contributes exact
// zeros to all three sums.  Entry e of the matrix is stored as
// m[3e], m[3e+1], m[3e+2] = c, d - c, c + d; every other k keeps (re, im) pairs.
template <int K> struct ThreeMult { static constexpr bool on = K == 4; };

// FP32 4-qubit gates compute two rows at once with the packed FP32 pair FMA of
// sm_100 (__ffma2_rn: two independent IEEE fmas in one instruction), halving
// the FMA instructions a pass issues; every lane performs the same fma sequence
// as the scalar form, so the results are bit-identical.  The 3M entries are
// then interleaved by row pair: for rows 2p, 2p+1 and column c the six floats
// at 6 (p D + c) are (c_0, c_1, (d-c)_0, (d-c)_1, (c+d)_0, (c+d)_1).
template <typename T, int K> struct PairedRows {
  static constexpr bool on = sizeof(T) == 4 && ThreeMult<K>::on;
};

template <typename T, int K> struct MatParam {
  __align__(8) T m[(ThreeMult<K>::on ? 3 : 2) * (1 << K) * (1 << K)];
};

// Row r of M times the D amplitudes x, for the register and tile kernels.
template <typename T, int K, typename V>
__device__ __forceinline__ V gate_row(const MatParam<T, K> &M, int r, const V (&x)[1 << K],
                                      const T (&sx)[1 << K]) {
  constexpr int D = 1 << K;
  V o;
  if constexpr (ThreeMult<K>::on) {
    T s1 = T(0), s2 = T(0), s3 = T(0);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      s1 = fma(M.m[3 * (r * D + c)], sx[c], s1);
      s2 = fma(M.m[3 * (r * D + c) + 1], x[c].x, s2);
      s3 = fma(M.m[3 * (r * D + c) + 2], x[c].y, s3);
    }
    o.x = s1 - s3;
    o.y = s1 + s2;
  } else {
    T re = T(0), im = T(0);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const T mr = M.m[2 * (r * D + c)];
      const T mi = M.m[2 * (r * D + c) + 1];
      re = fma(mr, x[c].x, re);
      re = fma(-mi, x[c].y, re);
      im = fma(mr, x[c].y, im);
      im = fma(mi, x[c].x, im);
    }
    o.x = re;
    o.y = im;
  }
  return o;
}

// Rows 2p and 2p + 1 of M times x in the paired FP32 3M form.
template <int K>
__device__ __forceinline__ void gate_row_pair(const MatParam<float, K> &M, int p,
                                              const float2 (&x)[1 << K], const float (&sx)[1 << K],
                                              float2 &o0, float2 &o1) {
  constexpr int D = 1 << K;
  float2 s1 = make_float2(0.f, 0.f), s2 = s1, s3 = s1;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const float2 *m = reinterpret_cast<const float2 *>(&M.m[6 * (p * D + c)]);
    s1 = __ffma2_rn(m[0], make_float2(sx[c], sx[c]), s1);
    s2 = __ffma2_rn(m[1], make_float2(x[c].x, x[c].x), s2);
    s3 = __ffma2_rn(m[2], make_float2(x[c].y, x[c].y), s3);
  }
  const float2 re = __fadd2_rn(s1, make_float2(-s3.x, -s3.y));
  const float2 im = __fadd2_rn(s1, s2);
  o0 = make_float2(re.x, im.x);
  o1 = make_float2(re.y, im.y);
}

// a + b of each amplitude, the shared operand of S1 (3M form only).
template <typename T, int K, typename V>
__device__ __forceinline__ void row_sums(const V (&x)[1 << K], T (&sx)[1 << K]) {
  if constexpr (ThreeMult<K>::on) {
#pragma unroll
    for (int c = 0; c < (1 << K); ++c) sx[c] = x[c].x + x[c].y;
  }
}

// Group index -> amplitude index of the group's first member: insert a zero
// bit at every target position, lowest first (the PDEP of cuda_gen.cpp:174-211).
template <int K>
__device__ __forceinline__ uint64_t group_base(uint64_t g, const Targets &t) {
#pragma unroll
  for (int b = 0; b < K; ++b) g = ((g & ~t.lo_mask[b]) << 1) | (g & t.lo_mask[b]);
  return g;
}

template <int K>
__device__ __forceinline__ uint64_t member_offset(int a, const Targets &t) {
  uint64_t off = 0;
#pragma unroll
  for (int b = 0; b < K; ++b)
    if ((a >> b) & 1) off += t.stride[b];
  return off;
}

// Register kernel: thread -> U gather groups (U = 2 for k <= 2 so that each
// thread keeps >= 64 bytes in flight), no grid-stride loop: a loop would let
// the compiler hoist the matrix out of the constant bank into registers.
constexpr int kRegThreads = 128;

template <int K> struct RegUnroll { static constexpr int U = K <= 2 ? 2 : 1; };

template <typename T, int K>
__global__ void __launch_bounds__(kRegThreads) k_gate_reg(T *__restrict__ sv, uint64_t n_groups,
                                                          Targets t, MatParam<T, K> M) {
  using V = typename Vec2<T>::type;
  constexpr int D = 1 << K;
  constexpr int U = RegUnroll<K>::U;
  V *psi = reinterpret_cast<V *>(sv);
  const uint64_t g0 = (uint64_t)blockIdx.x * (kRegThreads * U) + threadIdx.x;
  uint64_t base[U];
  V x[U][D];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const uint64_t g = g0 + (uint64_t)u * kRegThreads;
    base[u] = group_base<K>(g < n_groups ? g : 0, t);
    if (g < n_groups) {
#pragma unroll
      for (int a = 0; a < D; ++a) x[u][a] = psi[base[u] + member_offset<K>(a, t)];
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (g0 + (uint64_t)u * kRegThreads >= n_groups) break;
    T sx[D];
    row_sums<T, K>(x[u], sx);
    if constexpr (PairedRows<T, K>::on) {
#pragma unroll
      for (int p = 0; p < D / 2; ++p) {
        float2 o0, o1;
        gate_row_pair<K>(M, p, x[u], sx, o0, o1);
        psi[base[u] + member_offset<K>(2 * p, t)] = o0;
        psi[base[u] + member_offset<K>(2 * p + 1, t)] = o1;
      }
    } else {
#pragma unroll
      for (int r = 0; r < D; ++r) psi[base[u] + member_offset<K>(r, t)] = gate_row<T, K>(M, r, x[u], sx);
    }
  }
}

// Tile kernel for gates with targets among the low (intra-cache-line) qubits.
// A CTA owns one tile: the 2^(tb + k_hi) amplitudes whose "outer" bits are
// fixed, i.e. 2^k_hi chunks (one per combination of the targets >= tb) of
// 2^tb contiguous amplitudes.  The chunks are read with fully coalesced
// asynchronous copies (cp.async, the whole tile in flight, no register round
// trip) and written with coalesced 128/64-bit stores; the gate is applied inside
// shared memory,
// where the tile-local layout puts the high targets at bits tb..tb+k_hi-1.
// Shared memory is XOR-swizzled inside each 128-byte block so that both the
// contiguous phases and the strided gather of group members avoid bank
// conflicts.
template <int K> struct TileThreads { static constexpr int N = K <= 2 ? 256 : 128; };
constexpr int kTileMaxChunks = 1 << kMaxGateQubits;

struct TileArgs {
  uint64_t hi_lo_mask[kMaxGateQubits];   // (1 << hq_j) - 1 for the high targets
  uint64_t chunk_off[kTileMaxChunks];    // chunk c -> sum_j bit_j(c) << hq_j
  uint32_t loc_lo_mask[kMaxGateQubits];  // tile-local target positions (ascending) as masks
  uint32_t tb;                           // contiguous low bits per chunk
  uint32_t k_hi;                         // number of high targets
};

template <int LOGE>
__device__ __forceinline__ uint32_t swz(uint32_t i) {
  return i ^ ((i >> LOGE) & ((1u << LOGE) - 1));
}

// Built-in routing of dense k <= 4 gates with a target below qubit 5, per
// precision (FP32, FP64), k and the mask of those targets: 'r' the register
// kernel, 'a' the tile kernel with 2048 amplitudes a tile, 'b' with 4096 ('-'
// masks with more than k bits).  Measured on a B200 by the kernel autotuner
// (autotune kernels --n 30 --cxx-table: the fastest of the three on a
// Haar-random gate over a 30-qubit register, a tile kernel only where it beats
// the register kernel by more than 2%; the 26-qubit run picks kernels within 2%
// of these).  cast_b200_set_kernel_choice overrides it per class.
constexpr char kDefaultChoice[2][5][33] = {
    {"", "-rr-r---r-------r---------------", "-rrarrr-rrr-r---rrr-r---r-------", "-rrbrrrbrrrbrbb-rrrbrrr-rrr-r---", "-rrbrrrbrrrbrbbbrrrbrrrbrrrbrbb-"},
    {"", "-rr-r---r-------r---------------", "-rrbrar-rrr-r---rrr-r---r-------", "-rrbrbrbrrrbrbb-rrrrrbr-rrr-r---", "-rrrrrrarrrrrrrarrrrrrrarrrrrrr-"},
};

template <typename T, int K, int TB>
__global__ void __launch_bounds__(TileThreads<K>::N) k_gate_tile(T *__restrict__ sv, TileArgs a,
                                                                 MatParam<T, K> M) {
  constexpr int kTileThreads = TileThreads<K>::N;
  using V = typename Vec2<T>::type;
  constexpr int D = 1 << K;
  constexpr uint32_t TILE = 1u << TB;
  constexpr int LOGE = sizeof(V) == 16 ? 3 : 4;  // elements per 128-byte block
  // groups per thread, fully unrolled (a runtime loop would let the compiler
  // hoist the matrix out of the constant bank into registers)
  constexpr int GPT = (int)((TILE >> K) + kTileThreads - 1) / kTileThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *s = reinterpret_cast<V *>(smem_raw);
  V *psi = reinterpret_cast<V *>(sv);
  const uint32_t low_mask = (1u << a.tb) - 1;
  uint64_t tile_base = (uint64_t)blockIdx.x << a.tb;
  for (uint32_t j = 0; j < a.k_hi; ++j)
    tile_base = ((tile_base & ~a.hi_lo_mask[j]) << 1) | (tile_base & a.hi_lo_mask[j]);
  // asynchronous global -> shared copies: the whole tile in flight at once
  for (uint32_t i = threadIdx.x; i < TILE; i += kTileThreads)
    __pipeline_memcpy_async(&s[swz<LOGE>(i)], &psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)],
                            sizeof(V));
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
#pragma unroll
  for (int u = 0; u < GPT; ++u) {
    const uint32_t gl = threadIdx.x + u * kTileThreads;
    if (gl < (TILE >> K)) {
      uint32_t base = gl;
#pragma unroll
      for (int b = 0; b < K; ++b)
        base = ((base & ~a.loc_lo_mask[b]) << 1) | (base & a.loc_lo_mask[b]);
      V x[D];
#pragma unroll
      for (int m = 0; m < D; ++m) {
        uint32_t o = base;
#pragma unroll
        for (int b = 0; b < K; ++b)
          if ((m >> b) & 1) o += a.loc_lo_mask[b] + 1;
        x[m] = s[swz<LOGE>(o)];
      }
      T sx[D];
      row_sums<T, K>(x, sx);
      auto put = [&](int r, const V &o) {
        uint32_t po = base;
#pragma unroll
        for (int b = 0; b < K; ++b)
          if ((r >> b) & 1) po += a.loc_lo_mask[b] + 1;
        s[swz<LOGE>(po)] = o;
      };
      if constexpr (PairedRows<T, K>::on) {
#pragma unroll
        for (int p = 0; p < D / 2; ++p) {
          float2 o0, o1;
          gate_row_pair<K>(M, p, x, sx, o0, o1);
          put(2 * p, o0);
          put(2 * p + 1, o1);
        }
      } else {
#pragma unroll
        for (int r = 0; r < D; ++r) put(r, gate_row<T, K>(M, r, x, sx));
      }
    }
  }
  __syncthreads();
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < TILE; i += kTileThreads)
    psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)] = s[swz<LOGE>(i)];
}

// Staged kernel for k = 6, 7: a register-tiled complex GEMM per tile of G
// groups.  The CTA copies the tile's D x G amplitudes into shared memory with
// cp.async (coalesced: consecutive threads take consecutive groups of one
// member; every copy of the tile in flight at once, no register round trip),
// then thread (rs, gs) computes rows rs + i*RS (i < TR) for groups gs + j*GS
// (j < TG): per column c it loads TR matrix entries (the same for all lanes of
// a row slot: broadcast) and TG amplitudes (consecutive lanes, conflict-free)
// for TR*TG complex multiply-adds, so loads stay well below the FMA count.
// The matrix sits in shared memory when it takes at most 32 KB (FP32, k = 6),
// else it is read through L1.  Two CTAs a SM overlap one's copies with the
// other's arithmetic.  The products go straight back to HBM, the tile having
// been read in full.
constexpr int kStagedThreads = 256;

template <typename T, int K> struct StagedShape {
  static constexpr int D = 1 << K;
  static constexpr int TR = sizeof(T) == 4 ? 8 : 4;  // rows a thread
  static constexpr int TG = 4;                       // groups a thread
  static constexpr int RS = D / TR;                  // row slots
  static constexpr int GS = kStagedThreads / RS;     // group slots
  static constexpr int G = TG * GS;                  // groups a tile
  static constexpr bool kMatSmem = D * D * sizeof(T) * 2 <= 32768;  // matrix in shared memory
  static constexpr int MAT_SMEM = kMatSmem ? D * D : 0;             // its entries
  static_assert(RS * GS == kStagedThreads, "staged tile must use every thread");
};

template <typename T, int K>
__global__ void __launch_bounds__(kStagedThreads, 2) k_gate_staged(
    T *__restrict__ sv, uint64_t n_groups, Targets t, const typename Vec2<T>::type *__restrict__ mat) {
  using V = typename Vec2<T>::type;
  using Sh = StagedShape<T, K>;
  constexpr int D = Sh::D, TR = Sh::TR, TG = Sh::TG, RS = Sh::RS, GS = Sh::GS, G = Sh::G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *s = reinterpret_cast<V *>(smem_raw);  // [D][G]
  V *msm = s + D * G;
  V *psi = reinterpret_cast<V *>(sv);
  const int rs = threadIdx.x / GS, gs = threadIdx.x % GS;
  if constexpr (Sh::kMatSmem) {
    for (int i = threadIdx.x; i < D * D; i += kStagedThreads) msm[i] = mat[i];
  }
  const uint64_t n_tiles = (n_groups + G - 1) / G;
  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const uint64_t g0 = tile * G;
    // asynchronous global -> shared copies: every load of the tile in flight at once
    for (int i = threadIdx.x; i < D * G; i += kStagedThreads) {
      const int gg = i % G, a = i / G;
      const uint64_t g = g0 + gg;
      if (g < n_groups)
        __pipeline_memcpy_async(&s[a * G + gg], &psi[group_base<K>(g, t) + member_offset<K>(a, t)],
                                sizeof(V));
    }
    __pipeline_commit();
    __pipeline_wait_prior(0);
    __syncthreads();
    T re[TR][TG], im[TR][TG];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
      for (int j = 0; j < TG; ++j) re[i][j] = im[i][j] = T(0);
#pragma unroll 2
    for (int c = 0; c < D; ++c) {
      V x[TG];
#pragma unroll
      for (int j = 0; j < TG; ++j) x[j] = s[c * G + gs + j * GS];
#pragma unroll
      for (int i = 0; i < TR; ++i) {
        V m;
        if constexpr (Sh::kMatSmem) m = msm[(rs + i * RS) * D + c];
        else m = __ldg(&mat[(rs + i * RS) * D + c]);
#pragma unroll
        for (int j = 0; j < TG; ++j) {
          re[i][j] = fma(m.x, x[j].x, re[i][j]);
          re[i][j] = fma(-m.y, x[j].y, re[i][j]);
          im[i][j] = fma(m.x, x[j].y, im[i][j]);
          im[i][j] = fma(m.y, x[j].x, im[i][j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < TG; ++j) {
      const uint64_t g = g0 + gs + j * GS;
      if (g < n_groups) {
        const uint64_t base = group_base<K>(g, t);
#pragma unroll
        for (int i = 0; i < TR; ++i) {
          V o;
          o.x = re[i][j];
          o.y = im[i][j];
          psi[base + member_offset<K>(rs + i * RS, t)] = o;
        }
      }
    }
    __syncthreads();
  }
}

// Sparse kernel (k >= 5 with few nonzeros a row, e.g. fused CX / phase blocks
// of a QFT, which are monomial: one nonzero a row).  The reference's generator
// emits only the nonzero products of such a matrix (cuda_gen.cpp:223-284); here
// the matrix is a CSR table in device memory (values, row starts, columns).
// A CTA of 512 threads owns S strips of 32 consecutive groups.  The rows of a
// strip are split into W chunks of RPT = min(2^k, 16 (FP32) or 8 (FP64)) rows,
// one warp each, so
// lane l of a warp computes RPT rows of group l of its strip and every load and
// store of a warp covers 32 consecutive groups of one row (coalesced for high
// targets; for low ones L1 absorbs the gather).  The first nonzero of each of a
// thread's rows is fetched before any arithmetic: a monomial gate keeps RPT
// loads in flight a thread, as the dense register kernel does.  The CSR table
// and the 2^k member offsets are staged in shared memory once a CTA, so a row's
// bookkeeping is broadcast shared loads.  The CTA barrier between the reads and
// the in-place writes keeps every group's inputs intact until all its rows are
// computed.
// STAGED (gates with a row of more than one nonzero, e.g. the 4-nonzero blocks
// of a fused QFT): thread (chunk, lane) loads members r0 .. r0 + RPT - 1 of its
// group - every load in flight at once - into a [member][group] array in shared
// memory; after one barrier each row reads its inputs there (consecutive lanes,
// consecutive groups: no bank conflicts) instead of issuing a chain of
// dependent global loads per row.  64 KB a CTA in every shape.
// Shared memory of the sparse kernel: values, member offsets, row starts, columns.
__host__ __device__ inline size_t sparse_smem_bytes(uint32_t k, size_t v_bytes, uint32_t nnz) {
  return ((nnz * v_bytes + 15) & ~size_t(15)) + sizeof(uint64_t) * (1u << k) +
         sizeof(uint32_t) * ((1u << k) + 1 + nnz);
}

// Staging array of the STAGED sparse kernel: after the table, 16-byte aligned.
__host__ __device__ inline size_t sparse_stage_offset(uint32_t k, size_t v_bytes, uint32_t nnz) {
  return (sparse_smem_bytes(k, v_bytes, nnz) + 15) & ~size_t(15);
}

template <typename T, int K> struct SparseShape {
  static constexpr int THREADS = 512;
  static constexpr int D = 1 << K;
  static constexpr int MAX_RPT = sizeof(T) == 8 ? 8 : 16;  // 64 registers a thread
  static constexpr int RPT = D < MAX_RPT ? D : MAX_RPT;    // rows a thread
  static constexpr int W = D / RPT;            // row chunks (warps) a strip
  static constexpr int S = THREADS / 32 / W;   // strips a CTA
  static constexpr int G = 32 * S;             // groups a CTA
};

template <typename T, int K, bool STAGED>
__global__ void __launch_bounds__(SparseShape<T, K>::THREADS, 2) k_gate_sparse(
    T *__restrict__ sv, uint64_t n_groups, Targets t, const typename Vec2<T>::type *__restrict__ g_vals,
    const uint32_t *__restrict__ g_rows, const uint32_t *__restrict__ g_cols, uint32_t nnz) {
  using V = typename Vec2<T>::type;
  using Sh = SparseShape<T, K>;
  constexpr int D = 1 << K, RPT = Sh::RPT, W = Sh::W, G = Sh::G;
  // the CSR table and the member offsets, staged once a CTA (uniform reads)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *vals = reinterpret_cast<V *>(smem_raw);
  uint64_t *offs = reinterpret_cast<uint64_t *>(smem_raw + ((nnz * sizeof(V) + 15) & ~size_t(15)));
  uint32_t *row_start = reinterpret_cast<uint32_t *>(offs + D);
  uint32_t *cols = row_start + D + 1;
  for (uint32_t i = threadIdx.x; i < nnz; i += Sh::THREADS) {
    vals[i] = __ldg(&g_vals[i]);
    cols[i] = __ldg(&g_cols[i]);
  }
  for (uint32_t i = threadIdx.x; i <= (uint32_t)D; i += Sh::THREADS) {
    row_start[i] = __ldg(&g_rows[i]);
    if (i < (uint32_t)D) offs[i] = member_offset<K>((int)i, t);
  }
  __syncthreads();
  V *psi = reinterpret_cast<V *>(sv);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r0 = (w % W) * RPT;  // first row of this thread's chunk
  const uint64_t g = (uint64_t)blockIdx.x * G + (uint64_t)(w / W) * 32 + lane;
  const bool live = g < n_groups;
  const uint64_t base = group_base<K>(live ? g : 0, t);
  if constexpr (STAGED) {
    V *xs = reinterpret_cast<V *>(smem_raw + sparse_stage_offset(K, sizeof(V), nnz));  // [D][G]
    const int gl = (w / W) * 32 + lane;  // the group's column in the staging array
    V xin[RPT];
#pragma unroll
    for (int i = 0; i < RPT; ++i) xin[i] = live ? psi[base + offs[r0 + i]] : V{T(0), T(0)};
#pragma unroll
    for (int i = 0; i < RPT; ++i) xs[(r0 + i) * G + gl] = xin[i];
    __syncthreads();
    if (!live) return;
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const uint32_t a = row_start[r0 + i], e = row_start[r0 + i + 1];
      T re = T(0), im = T(0);
      if (a < e) {
        V m = vals[a];
        V x = xs[cols[a] * G + gl];
        re = fma(m.x, x.x, -m.y * x.y);
        im = fma(m.x, x.y, m.y * x.x);
        for (uint32_t j = a + 1; j < e; ++j) {
          m = vals[j];
          x = xs[cols[j] * G + gl];
          re = fma(m.x, x.x, fma(-m.y, x.y, re));
          im = fma(m.x, x.y, fma(m.y, x.x, im));
        }
      }
      V o;
      o.x = re;
      o.y = im;
      psi[base + offs[r0 + i]] = o;
    }
    return;
  }
  uint32_t js[RPT], je[RPT];
  V x0[RPT];
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    js[i] = row_start[r0 + i];
    je[i] = row_start[r0 + i + 1];
    if (live && js[i] < je[i]) x0[i] = psi[base + offs[cols[js[i]]]];
  }
  T re[RPT], im[RPT];
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    re[i] = im[i] = T(0);
    if (!live || js[i] >= je[i]) continue;
    V m = vals[js[i]];
    re[i] = fma(m.x, x0[i].x, -m.y * x0[i].y);
    im[i] = fma(m.x, x0[i].y, m.y * x0[i].x);
    for (uint32_t j = js[i] + 1; j < je[i]; ++j) {
      m = vals[j];
      const V x = psi[base + offs[cols[j]]];
      re[i] = fma(m.x, x.x, fma(-m.y, x.y, re[i]));
      im[i] = fma(m.x, x.y, fma(m.y, x.x, im[i]));
    }
  }
  __syncthreads();
  if (live) {
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      V o;
      o.x = re[i];
      o.y = im[i];
      psi[base + offs[r0 + i]] = o;
    }
  }
}

// Sparse gate with targets among the low qubits: the tile kernel's geometry
// (tile_geometry, whole groups inside a tile of 2048 amplitudes) with the CSR
// arithmetic.  The tile is copied in with cp.async; thread t computes tile
// amplitudes t, t + 512, ...: row r = the target bits of the tile-local index,
// inputs read from shared memory at the group base plus the tile-local member
// offsets of the row's columns.  After a barrier the outputs go back into the
// tile and the tile is stored coalesced.
constexpr int kSparseTileThreads = 512;

template <typename T, int K, int TB>
__global__ void __launch_bounds__(kSparseTileThreads) k_gate_sparse_tile(
    T *__restrict__ sv, TileArgs a, const typename Vec2<T>::type *__restrict__ g_vals,
    const uint32_t *__restrict__ g_rows, const uint32_t *__restrict__ g_cols, uint32_t nnz) {
  using V = typename Vec2<T>::type;
  constexpr int D = 1 << K;
  constexpr uint32_t TILE = 1u << TB;
  constexpr int OPT = TILE / kSparseTileThreads;  // outputs a thread
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *tile = reinterpret_cast<V *>(smem_raw);
  V *vals = tile + TILE;
  uint32_t *offs = reinterpret_cast<uint32_t *>(smem_raw + sizeof(V) * TILE +
                                                ((nnz * sizeof(V) + 15) & ~size_t(15)));
  uint32_t *row_start = offs + D;
  uint32_t *cols = row_start + D + 1;
  V *psi = reinterpret_cast<V *>(sv);
  const uint32_t low_mask = (1u << a.tb) - 1;
  uint64_t tile_base = (uint64_t)blockIdx.x << a.tb;
  for (uint32_t j = 0; j < a.k_hi; ++j)
    tile_base = ((tile_base & ~a.hi_lo_mask[j]) << 1) | (tile_base & a.hi_lo_mask[j]);
  if constexpr (sizeof(V) == 8) {
    // FP32: amplitude pairs (a chunk is a contiguous run of >= 32 amplitudes
    // starting at an even index) as 16-byte copies
    for (uint32_t i = 2 * threadIdx.x; i < TILE; i += 2 * kSparseTileThreads)
      __pipeline_memcpy_async(&tile[i], &psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)], 16);
  } else {
    for (uint32_t i = threadIdx.x; i < TILE; i += kSparseTileThreads)
      __pipeline_memcpy_async(&tile[i], &psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)],
                              sizeof(V));
  }
  __pipeline_commit();
  uint32_t tmask = 0;  // tile-local target bits
#pragma unroll
  for (int b = 0; b < K; ++b) tmask |= a.loc_lo_mask[b] + 1;
  for (uint32_t i = threadIdx.x; i < nnz; i += kSparseTileThreads) {
    vals[i] = __ldg(&g_vals[i]);
    cols[i] = __ldg(&g_cols[i]);
  }
  for (uint32_t i = threadIdx.x; i <= (uint32_t)D; i += kSparseTileThreads) {
    row_start[i] = __ldg(&g_rows[i]);
    if (i < (uint32_t)D) {
      uint32_t o = 0;
#pragma unroll
      for (int b = 0; b < K; ++b)
        if ((i >> b) & 1) o += a.loc_lo_mask[b] + 1;
      offs[i] = o;
    }
  }
  __pipeline_wait_prior(0);
  __syncthreads();
  V out[OPT];
#pragma unroll
  for (int u = 0; u < OPT; ++u) {
    const uint32_t o = threadIdx.x + u * kSparseTileThreads;
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < K; ++b) r |= ((o & (a.loc_lo_mask[b] + 1)) != 0) << b;
    const uint32_t gb = o & ~tmask;
    T re = T(0), im = T(0);
    for (uint32_t j = row_start[r]; j < row_start[r + 1]; ++j) {
      const V m = vals[j];
      const V x = tile[gb + offs[cols[j]]];
      re = fma(m.x, x.x, fma(-m.y, x.y, re));
      im = fma(m.x, x.y, fma(m.y, x.x, im));
    }
    out[u].x = re;
    out[u].y = im;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < OPT; ++u) tile[threadIdx.x + u * kSparseTileThreads] = out[u];
  __syncthreads();
  if constexpr (sizeof(V) == 8) {
    for (uint32_t i = 2 * threadIdx.x; i < TILE; i += 2 * kSparseTileThreads)
      *reinterpret_cast<float4 *>(&psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)]) =
          *reinterpret_cast<const float4 *>(&tile[i]);
  } else {
    for (uint32_t i = threadIdx.x; i < TILE; i += kSparseTileThreads)
      psi[tile_base + a.chunk_off[i >> a.tb] + (i & low_mask)] = tile[i];
  }
}

// Device CSR table of a sparse gate: values (interleaved, the gate's
// precision), then D + 1 row starts, then the column of every value.
struct SparseLayout {
  size_t row_off = 0, col_off = 0, bytes = 0;
};

SparseLayout sparse_layout(uint32_t k, uint8_t precision, size_t nnz) {
  auto align16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  SparseLayout l;
  l.row_off = align16(nnz * 2 * (precision ? sizeof(double) : sizeof(float)));
  l.col_off = align16(l.row_off + sizeof(uint32_t) * ((1u << k) + 1));
  l.bytes = l.col_off + sizeof(uint32_t) * std::max<size_t>(nnz, 1);
  return l;
}

// Largest number of nonzeros in one row of the gate.
size_t gate_row_nnz_max(const GateData &g) {
  const size_t d = size_t(1) << g.k;
  size_t best = 0;
  for (size_t r = 0; r < d; ++r) {
    size_t c = 0;
    for (size_t e = r * d; e < (r + 1) * d; ++e) c += g.m64[2 * e] != 0.0 || g.m64[2 * e + 1] != 0.0;
    best = std::max(best, c);
  }
  return best;
}

size_t gate_nnz(const GateData &g) {
  size_t nnz = 0;
  for (size_t e = 0; e < g.m64.size() / 2; ++e) nnz += g.m64[2 * e] != 0.0 || g.m64[2 * e + 1] != 0.0;
  return nnz;
}

int g_sm_count = 0;
std::once_flag g_sm_once;

template <typename F> int max_blocks_per_sm(F kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess ||
      b < 1)
    b = 1;
  return b;
}

// The kernel-parameter copy of the matrix: the snapped (re, im) pairs as they
// are, or for the 3M form (c, d - c, c + d) per entry, formed in FP64 from the
// snapped matrix and rounded once to T.  The launch copies the parameters, so
// `scratch` only has to outlive the launch call.
template <typename T, int K>
const MatParam<T, K> *mat_param(const GateData &g, MatParam<T, K> &scratch) {
  if constexpr (ThreeMult<K>::on) {
    constexpr size_t E = size_t(1) << (2 * K);
    const bool wide = g.m64.size() == 2 * E;
    constexpr size_t D = size_t(1) << K;
    for (size_t e = 0; e < E; ++e) {
      const double c = wide ? g.m64[2 * e] : (double)g.m32[2 * e];
      const double d = wide ? g.m64[2 * e + 1] : (double)g.m32[2 * e + 1];
      // scalar form: entry e at 3e; paired form: see PairedRows
      const size_t r = e / D, col = e % D;
      const size_t at = PairedRows<T, K>::on ? 6 * ((r / 2) * D + col) + (r & 1) : 3 * e;
      const size_t step = PairedRows<T, K>::on ? 2 : 1;
      scratch.m[at] = (T)c;
      scratch.m[at + step] = (T)(d - c);
      scratch.m[at + 2 * step] = (T)(c + d);
    }
    return &scratch;
  } else {
    (void)scratch;
    if constexpr (sizeof(T) == 8) return reinterpret_cast<const MatParam<T, K> *>(g.m64.data());
    else return reinterpret_cast<const MatParam<T, K> *>(g.m32.data());
  }
}

template <typename T, int K>
bool launch_reg(const GateData &g, void *sv, uint32_t n, const Targets &t, cudaStream_t s,
                std::string &err) {
  constexpr int U = RegUnroll<K>::U;
  const uint64_t n_groups = 1ull << (n - K);
  const uint64_t blocks = (n_groups + kRegThreads * U - 1) / (kRegThreads * U);
  if (blocks > 0x7fffffffull) {
    err = "statevector too large for the gate kernel grid";
    return false;
  }
  MatParam<T, K> scratch;
  const MatParam<T, K> *mp = mat_param<T, K>(g, scratch);
  T *p = static_cast<T *>(sv);
  void *args[] = {&p, const_cast<uint64_t *>(&n_groups), const_cast<Targets *>(&t),
                  const_cast<MatParam<T, K> *>(mp)};
  return cuda_ok(cudaLaunchKernel((const void *)k_gate_reg<T, K>, dim3((unsigned)blocks),
                                  dim3(kRegThreads), args, 0, s),
                 "gate kernel launch", err);
}

template <typename T, int K>
bool launch_sparse(const GateData &g, void *sv, uint32_t n, const Targets &t, cudaStream_t s,
                   std::string &err) {
  using V = typename Vec2<T>::type;
  const SparseLayout l = sparse_layout(K, g.precision, gate_nnz(g));
  const char *base = static_cast<const char *>(g.d_sparse);
  const uint64_t n_groups = 1ull << (n - K);
  constexpr int G = SparseShape<T, K>::G;  // groups a CTA
  const uint64_t blocks = (n_groups + G - 1) / G;
  if (blocks > 0x7fffffffull) {
    err = "statevector too large for the sparse gate kernel grid";
    return false;
  }
  const uint32_t nnz = (uint32_t)gate_nnz(g);
  constexpr size_t kStage = sizeof(V) * SparseShape<T, K>::G * (1u << K);
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  std::call_once(once, [] {  // the largest table: 2^(2k) / 4 entries
    const uint32_t most = 1u << (2 * K - 2);
    attr_rc = cudaFuncSetAttribute(k_gate_sparse<T, K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sparse_smem_bytes(K, sizeof(V), most));
    if (attr_rc == cudaSuccess)
      attr_rc = cudaFuncSetAttribute(k_gate_sparse<T, K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sparse_stage_offset(K, sizeof(V), most) + kStage));
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(sparse gate kernel)", err)) return false;
  const V *vals = reinterpret_cast<const V *>(base);
  const uint32_t *rows = reinterpret_cast<const uint32_t *>(base + l.row_off);
  const uint32_t *cols = reinterpret_cast<const uint32_t *>(base + l.col_off);
  if (gate_row_nnz_max(g) > 1)
    k_gate_sparse<T, K, true><<<(unsigned)blocks, SparseShape<T, K>::THREADS,
                                sparse_stage_offset(K, sizeof(V), nnz) + kStage, s>>>(
        static_cast<T *>(sv), n_groups, t, vals, rows, cols, nnz);
  else
    k_gate_sparse<T, K, false><<<(unsigned)blocks, SparseShape<T, K>::THREADS,
                                 sparse_smem_bytes(K, sizeof(V), nnz), s>>>(
        static_cast<T *>(sv), n_groups, t, vals, rows, cols, nnz);
  return cuda_ok(cudaGetLastError(), "sparse gate kernel launch", err);
}

bool tile_geometry(const GateData &g, uint32_t n, TileArgs &a, uint32_t target);

// Tile of the sparse tile kernel: 4096 amplitudes in FP32 (32 KB), 2048 in FP64.
template <typename T> constexpr uint32_t sparse_tile_bits() { return sizeof(T) == 4 ? 12u : 11u; }

size_t sparse_tile_smem_bytes(uint32_t k, size_t v_bytes, uint32_t nnz, uint32_t tb) {
  return (v_bytes << tb) + ((nnz * v_bytes + 15) & ~size_t(15)) +
         sizeof(uint32_t) * (2 * (1u << k) + 1 + nnz);
}

template <typename T, int K>
bool launch_sparse_tile(const GateData &g, void *sv, uint32_t n, const TileArgs &a, cudaStream_t s,
                        std::string &err) {
  using V = typename Vec2<T>::type;
  const uint32_t nnz = (uint32_t)gate_nnz(g);
  const SparseLayout l = sparse_layout(K, g.precision, nnz);
  const char *base = static_cast<const char *>(g.d_sparse);
  constexpr uint32_t TB = sparse_tile_bits<T>();
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  std::call_once(once, [] {  // the largest table: 2^(2k) / 4 entries
    attr_rc = cudaFuncSetAttribute(k_gate_sparse_tile<T, K, TB>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sparse_tile_smem_bytes(K, sizeof(V), 1u << (2 * K - 2), TB));
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(sparse tile kernel)", err)) return false;
  const uint64_t n_tiles = 1ull << (n - TB);
  k_gate_sparse_tile<T, K, TB><<<(unsigned)n_tiles, kSparseTileThreads,
                                 sparse_tile_smem_bytes(K, sizeof(V), nnz, TB), s>>>(
      static_cast<T *>(sv), a, reinterpret_cast<const V *>(base),
      reinterpret_cast<const uint32_t *>(base + l.row_off),
      reinterpret_cast<const uint32_t *>(base + l.col_off), nnz);
  return cuda_ok(cudaGetLastError(), "sparse tile kernel launch", err);
}

// Sparse gates with a target below qubit 5 run tiled (a warp's direct loads
// would each gather from 32 groups 2^k amplitudes apart); the others read
// global memory directly.
bool sparse_tile_chosen(const GateData &g, uint32_t n, TileArgs &a) {
  if (g.qubits[0] >= 5) return false;
  std::memset(&a, 0, sizeof(a));
  return tile_geometry(g, n, a, g.precision == 1 ? sparse_tile_bits<double>() : sparse_tile_bits<float>());
}

template <typename T>
bool launch_sparse_t(const GateData &g, void *sv, uint32_t n, const Targets &t, cudaStream_t s,
                     std::string &err) {
  {
    TileArgs a;
    if (sparse_tile_chosen(g, n, a)) {
      switch (g.k) {
      case 5: return launch_sparse_tile<T, 5>(g, sv, n, a, s, err);
      case 6: return launch_sparse_tile<T, 6>(g, sv, n, a, s, err);
      case 7: return launch_sparse_tile<T, 7>(g, sv, n, a, s, err);
      default: break;
      }
    }
  }
  switch (g.k) {
  case 5: return launch_sparse<T, 5>(g, sv, n, t, s, err);
  case 6: return launch_sparse<T, 6>(g, sv, n, t, s, err);
  case 7: return launch_sparse<T, 7>(g, sv, n, t, s, err);
  default: err = "sparse kernel handles 5..7 qubits"; return false;
  }
}

// Tile geometry for a gate: returns false when the tile kernel does not apply.
bool tile_geometry(const GateData &g, uint32_t n, TileArgs &a, uint32_t target) {
  if (n < target) return false;
  uint32_t need = 0;  // every target below 5 must sit inside a chunk
  for (uint32_t b = 0; b < g.k; ++b)
    if (g.qubits[b] < 5) need = std::max(need, g.qubits[b] + 1);
  need = std::max<uint32_t>(need, 5);
  for (uint32_t tb = target; tb >= need; --tb) {
    uint32_t khi = 0;
    for (uint32_t b = 0; b < g.k; ++b) khi += g.qubits[b] >= tb;
    if (tb + khi > target) continue;
    a.tb = tb;
    a.k_hi = khi;
    uint32_t j = 0;
    uint32_t hq[kMaxGateQubits] = {0};
    for (uint32_t b = 0; b < g.k; ++b) {
      if (g.qubits[b] >= tb) {
        hq[j] = g.qubits[b];
        a.hi_lo_mask[j] = (1ull << g.qubits[b]) - 1;
        ++j;
      }
    }
    // tile-local positions: low targets keep their bit, high target j -> tb + j
    uint32_t h = 0;
    for (uint32_t b = 0; b < g.k; ++b) {
      const uint32_t pos = g.qubits[b] < tb ? g.qubits[b] : tb + h++;
      a.loc_lo_mask[b] = (1u << pos) - 1;
    }
    for (uint32_t c = 0; c < (1u << khi); ++c) {
      uint64_t o = 0;
      for (uint32_t jj = 0; jj < khi; ++jj)
        if ((c >> jj) & 1) o += 1ull << hq[jj];
      a.chunk_off[c] = o;
    }
    return true;
  }
  return false;
}

template <typename T, int K, int TB>
bool launch_tile_tb(const GateData &g, void *sv, uint32_t n, const TileArgs &a, cudaStream_t s,
                    std::string &err) {
  using V = typename Vec2<T>::type;
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  std::call_once(once, [] {
    attr_rc = cudaFuncSetAttribute(k_gate_tile<T, K, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(V) << TB));
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(tile gate kernel)", err)) return false;
  const uint64_t n_tiles = 1ull << (n - TB);
  const size_t smem = sizeof(V) << TB;
  MatParam<T, K> scratch;
  const MatParam<T, K> *mp = mat_param<T, K>(g, scratch);
  T *p = static_cast<T *>(sv);
  void *args[] = {&p, const_cast<TileArgs *>(&a), const_cast<MatParam<T, K> *>(mp)};
  return cuda_ok(cudaLaunchKernel((const void *)k_gate_tile<T, K, TB>, dim3((unsigned)n_tiles),
                                  dim3(TileThreads<K>::N), args, smem, s),
                 "tile gate kernel launch", err);
}

template <typename T, int K>
bool launch_tile(const GateData &g, void *sv, uint32_t n, const TileArgs &a, cudaStream_t s,
                 std::string &err) {
  return a.tb + a.k_hi == 12 ? launch_tile_tb<T, K, 12>(g, sv, n, a, s, err)
                             : launch_tile_tb<T, K, 11>(g, sv, n, a, s, err);
}

template <typename T, int K>
bool launch_staged(const GateData &g, void *sv, uint32_t n, const Targets &t, cudaStream_t s,
                   std::string &err) {
  using V = typename Vec2<T>::type;
  constexpr int G = StagedShape<T, K>::G;
  constexpr size_t smem = sizeof(V) * ((1 << K) * G + StagedShape<T, K>::MAT_SMEM);
  static int blocks_per_sm = 0;
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  std::call_once(once, [] {
    attr_rc = cudaFuncSetAttribute(k_gate_staged<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem);
    blocks_per_sm = max_blocks_per_sm(k_gate_staged<T, K>, kStagedThreads, smem);
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(staged gate kernel)", err)) return false;
  if (!g.d_mat) {
    err = "staged gate kernel needs a device matrix";
    return false;
  }
  const uint64_t n_groups = 1ull << (n - K);
  const uint64_t n_tiles = (n_groups + G - 1) / G;
  const uint64_t cap = (uint64_t)blocks_per_sm * sm_count();
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(n_tiles, cap));
  k_gate_staged<T, K><<<grid, kStagedThreads, smem, s>>>(static_cast<T *>(sv), n_groups, t,
                                                          static_cast<const V *>(g.d_mat));
  return cuda_ok(cudaGetLastError(), "staged gate kernel launch", err);
}

// Path selection between the register and tile kernels (k <= 4);
// CAST_B200_GATE_PATH=reg|tile forces one path for measurement.
std::atomic<int> g_gate_path{[] {
  const char *e = std::getenv("CAST_B200_GATE_PATH");
  if (!e) return 0;
  if (!std::strcmp(e, "reg")) return 1;
  if (!std::strcmp(e, "tile")) return 2;
  return 0;
}()};

int gate_path_override() { return g_gate_path.load(std::memory_order_relaxed); }

// Per-class kernel choices written by the autotuner (cast_b200_set_kernel_choice).
// A class is (precision, k = 1..4, the mask of targets below qubit 5).  engine:
// -1 the built-in rule below, 0 register kernel, 1 tile kernel; tile_bits: 0 the
// built-in size, 11 or 12 (2048 / 4096 amplitudes a tile).
struct KernelChoice {
  std::atomic<int> engine{-1};
  std::atomic<int> tile_bits{0};
};
KernelChoice g_choice[2][5][32];

bool tile_chosen(const GateData &g, uint32_t n, TileArgs &a) {
  if (g.k > 4) return false;
  const int ov = gate_path_override();
  if (ov == 1) return false;
  uint32_t low_bits = 0;
  for (uint32_t b = 0; b < g.k; ++b)
    if (g.qubits[b] < 5) low_bits |= 1u << g.qubits[b];
  if (low_bits == 0) return false;
  const int p = g.precision ? 1 : 0;
  const char def = kDefaultChoice[p][g.k][low_bits];
  bool tile = def == 'a' || def == 'b';
  int tb = def == 'b' ? 12 : 11;
  const KernelChoice &c = g_choice[p][g.k][low_bits];
  const int tuned = c.engine.load(std::memory_order_relaxed);
  if (tuned >= 0) tile = tuned == 1;
  const int tuned_tb = c.tile_bits.load(std::memory_order_relaxed);
  if (tuned_tb == 11 || tuned_tb == 12) tb = tuned_tb;
  if (ov != 2 && !tile) return false;
  std::memset(&a, 0, sizeof(a));
  return tile_geometry(g, n, a, (uint32_t)tb);
}

template <typename T>
bool try_tile(const GateData &g, void *sv, uint32_t n, cudaStream_t s, std::string &err,
              bool &done) {
  done = false;
  TileArgs a;
  if (!tile_chosen(g, n, a)) return true;
  done = true;
  switch (g.k) {
  case 1: return launch_tile<T, 1>(g, sv, n, a, s, err);
  case 2: return launch_tile<T, 2>(g, sv, n, a, s, err);
  case 3: return launch_tile<T, 3>(g, sv, n, a, s, err);
  case 4: return launch_tile<T, 4>(g, sv, n, a, s, err);
  default: done = false; return true;
  }
}

template <typename T>
bool launch_t(const GateData &g, void *sv, uint32_t n, const Targets &t, cudaStream_t s,
              std::string &err) {
  bool done = false;
  if (!try_tile<T>(g, sv, n, s, err, done)) return false;
  if (done) return true;
  switch (g.k) {
  case 1: return launch_reg<T, 1>(g, sv, n, t, s, err);
  case 2: return launch_reg<T, 2>(g, sv, n, t, s, err);
  case 3: return launch_reg<T, 3>(g, sv, n, t, s, err);
  case 4: return launch_reg<T, 4>(g, sv, n, t, s, err);
  case 5: return launch_reg<T, 5>(g, sv, n, t, s, err);
  case 6: return launch_staged<T, 6>(g, sv, n, t, s, err);
  case 7: return launch_staged<T, 7>(g, sv, n, t, s, err);
  default: err = "unsupported gate size"; return false;
  }
}

}  // namespace

int set_gate_path(int path) { return g_gate_path.exchange(path < 0 || path > 2 ? 0 : path); }

bool set_kernel_choice(uint8_t precision, uint32_t k, uint32_t low_mask, int engine,
                       uint32_t tile_bits_, std::string &err) {
  if (precision > 1 || k < 1 || k > 4 || low_mask == 0 || low_mask > 31 ||
      (uint32_t)__builtin_popcount(low_mask) > k || engine < -1 || engine > 1 ||
      (tile_bits_ != 0 && tile_bits_ != 11 && tile_bits_ != 12)) {
    err = "kernel choice: precision 0/1, k 1..4, low mask 1..31 with at most k bits, engine "
          "-1/0/1, tile bits 0/11/12";
    return false;
  }
  KernelChoice &c = g_choice[precision][k][low_mask];
  c.engine.store(engine);
  c.tile_bits.store((int)tile_bits_);
  return true;
}

int sm_count() {
  std::call_once(g_sm_once, [] {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        g_sm_count < 1)
      g_sm_count = 1;
  });
  return g_sm_count;
}

bool check_gate(const GateData &g, uint32_t n, std::string &err) {
  if (g.k == 0 || g.k > kMaxGateQubits) {
    err = "gate must act on 1.." + std::to_string(kMaxGateQubits) + " qubits, got " +
          std::to_string(g.k);
    return false;
  }
  if (n < g.k) {
    err = "statevector has fewer qubits than the gate kernel requires";
    return false;
  }
  if (n > kMaxSvQubits) {
    err = "statevector qubit count " + std::to_string(n) + " exceeds the supported maximum";
    return false;
  }
  for (uint32_t b = 0; b < g.k; ++b) {
    if (g.qubits[b] >= n) {
      err = "gate acts on qubit " + std::to_string(g.qubits[b]) + " outside the " +
            std::to_string(n) + "-qubit statevector";
      return false;
    }
    if (b && g.qubits[b - 1] >= g.qubits[b]) {
      err = "gate qubits must be distinct and ascending";
      return false;
    }
  }
  const size_t want = 2ull << (2 * g.k);
  if ((g.precision == 1 && g.m64.size() != want) || (g.precision == 0 && g.m32.size() != want)) {
    err = "gate matrix has the wrong size";
    return false;
  }
  return true;
}

bool launch_gate(const GateData &g, void *sv, uint32_t n, cudaStream_t stream, std::string &err) {
  if (!check_gate(g, n, err)) return false;
  if (!sv) {
    err = "statevector pointer must not be null";
    return false;
  }
  if (!aligned16(reinterpret_cast<uint64_t>(sv), "statevector pointer", err)) return false;
  if (g.d_tc) return launch_gate_tensor(g, sv, n, stream, err);
  Targets t;
  for (uint32_t b = 0; b < kMaxGateQubits; ++b) {
    const uint32_t q = b < g.k ? g.qubits[b] : 0;
    t.lo_mask[b] = (1ull << q) - 1;
    t.stride[b] = 1ull << q;
  }
  if (g.d_sparse)
    return g.precision == 1 ? launch_sparse_t<double>(g, sv, n, t, stream, err)
                            : launch_sparse_t<float>(g, sv, n, t, stream, err);
  return g.precision == 1 ? launch_t<double>(g, sv, n, t, stream, err)
                          : launch_t<float>(g, sv, n, t, stream, err);
}

int gate_engine(const GateData &g, uint32_t n, bool tensor, bool sparse) {
  if (tensor) return kEngineTensor;
  TileArgs a;
  if (sparse) return sparse_tile_chosen(g, n, a) ? kEngineSparseTile : kEngineSparse;
  if (tile_chosen(g, n, a)) return kEngineTile;
  return g.k >= 6 ? kEngineStaged : kEngineRegister;
}

// Only from k = 5: below that the dense kernels are bound by HBM, not the FMA
// pipes, and beat the sparse kernel (FP32 monomial k = 3 on high targets: 4.5
// against 6.8 TB/s).
bool sparse_gate(const GateData &g) {
  if (g.k < 5 || g.k > kMaxGateQubits || g.m64.size() != (2ull << (2 * g.k))) return false;
  const size_t d = 1ull << g.k;
  return gate_nnz(g) * 4 <= d * d;
}

bool upload_sparse(GateData &g, std::string &err) {
  const uint32_t d = 1u << g.k;
  const size_t nnz = gate_nnz(g);
  const SparseLayout l = sparse_layout(g.k, g.precision, nnz);
  std::vector<unsigned char> host(l.bytes, 0);
  uint32_t *rows = reinterpret_cast<uint32_t *>(host.data() + l.row_off);
  uint32_t *cols = reinterpret_cast<uint32_t *>(host.data() + l.col_off);
  size_t j = 0;
  for (uint32_t r = 0; r < d; ++r) {
    rows[r] = (uint32_t)j;
    for (uint32_t c = 0; c < d; ++c) {
      const size_t e = (size_t)r * d + c;
      const double re = g.m64[2 * e], im = g.m64[2 * e + 1];
      if (re == 0.0 && im == 0.0) continue;
      if (g.precision) {
        reinterpret_cast<double *>(host.data())[2 * j] = re;
        reinterpret_cast<double *>(host.data())[2 * j + 1] = im;
      } else {
        reinterpret_cast<float *>(host.data())[2 * j] = g.m32[2 * e];
        reinterpret_cast<float *>(host.data())[2 * j + 1] = g.m32[2 * e + 1];
      }
      cols[j++] = c;
    }
  }
  rows[d] = (uint32_t)j;
  if (g.d_sparse) cudaFree(g.d_sparse);
  g.d_sparse = nullptr;
  if (!cuda_ok(cudaMalloc(&g.d_sparse, l.bytes), "cudaMalloc (sparse gate)", err)) return false;
  if (!cuda_ok(cudaMemcpy(g.d_sparse, host.data(), l.bytes, cudaMemcpyHostToDevice),
               "cudaMemcpy (sparse gate)", err)) {
    cudaFree(g.d_sparse);
    g.d_sparse = nullptr;
    return false;
  }
  return true;
}

void free_gate_device(GateData &g) {
  if (g.d_mat) cudaFree(g.d_mat);
  if (g.d_tc) cudaFree(g.d_tc);
  if (g.d_sparse) cudaFree(g.d_sparse);
  g.d_mat = g.d_tc = g.d_sparse = nullptr;
}

void snap_matrix(GateData &g, const double *m, double ztol, double otol) {
  const size_t dim = 1ull << g.k;
  const double K = (double)dim;
  const double zt = ztol / K, ot = otol / K;
  const size_t ns = 2 * dim * dim;
  g.m64.resize(ns);
  g.m32.resize(ns);
  for (size_t i = 0; i < ns; ++i) {
    const double v = m[i];
    double s;
    if (ztol > 0.0 && std::fabs(v) < zt) s = 0.0;
    else if (otol > 0.0 && std::fabs(v - 1.0) < ot) s = 1.0;
    else if (otol > 0.0 && std::fabs(v + 1.0) < ot) s = -1.0;
    else s = v;
    g.m64[i] = s;
    g.m32[i] = (float)s;
  }
}

}  // namespace cb2
