// Tensor-core gate application for complex64 statevectors, k = 5, 6, on the
// fifth-generation tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// A fused k-qubit gate M = A + iB (D x D, D = 2^k) applied to the gather groups
// of a statevector is a real GEMM with R = 2D reals per group.  It is issued
// transposed, one tile of 128 groups at a time:
//
//     Y^T (128 x R)  =  X^T (128 x R) . Mr^T,     Mr[2r+c'][2m+c] = the real
//     2x2 block [[A, -B], [B, A]] of M[r][m] (c, c' = 0 real, 1 imaginary),
//
// so the tile's groups are the MMA's M = 128 rows (one tensor-memory lane per
// group), the gate is the resident N x K = R x R operand, and the k16 loop runs
// over the group's members (Re, Im interleaved, exactly as the amplitudes lie in
// memory).  Every FP32 operand v is split into BF16 hi + lo (hi = bf16(v),
// lo = bf16(v - hi)) and Y = X_lo M_hi + X_hi M_lo + X_hi M_hi is accumulated in
// FP32 in tensor memory (the lo*lo term, below 2^-16 of the product, is
// dropped): about 2^-16 relative error per product, ~1e-5 of the group norm per
// fused pass.
//
// One persistent CTA per SM, warp-specialised:
//   warps 0-3   epilogue: tensor memory -> registers (tcgen05.ld 32x32b, lane =
//               group) -> coalesced 8-byte stores, 32 consecutive groups of one
//               member per warp instruction;
//   warps 4-15  loaders: 8-byte global loads of 4 members per (group, chunk),
//               split into BF16 hi/lo in registers and written with tcgen05.st
//               straight into tensor memory, where the MMA takes its A operand
//               (tcgen05.mma with [a_tmem]): the tile's 128 groups are the 128
//               lanes, and a 32-member K atom (one stage) is 32 columns of hi and
//               32 of lo, two BF16 a column with the even K index in the low half.
//               Loader warp w writes lanes 32 (w % 4) .. +31, the groups it loads;
//   warp 16     allocates tensor memory and issues the MMAs (one thread).
// A tile takes 2^k / 32 consecutive stages.  The loader warps form 3 groups of
// 128 threads that fill 4 A stages in rotation (group j takes stages j, j + 3,
// ...), each group issuing its next stage's loads before it waits for a free
// stage, so three stages of loads (96 KB) are in flight per SM.  Shared memory
// holds only the split gate (the MMA's B operand, 64 KB for k = 6) and
// bookkeeping: it is carved from the same array as the L1 that holds the loads
// in flight, and with the data operand in tensor memory instead of in shared
// stages a 6-qubit pass at 30 qubits went from 3.47 to 2.82 ms.  Tensor memory
// (512 columns): two accumulators, so the epilogue of one tile overlaps the MMAs
// of the next, and the four A stages.  Every wait on an mbarrier is bounded: on
// expiry the CTA records an error code (read back by tensor_error_status),
// drains its outstanding MMAs, frees its tensor memory and exits.
#include "internal.hpp"

#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <mutex>

namespace cb2 {

namespace {

constexpr int kTileGroups = 128;                   // MMA M: one TMEM lane per group
constexpr int kEpiWarps = 4;                       // warps 0-3 (TMEM sub-partitions 0-3)
constexpr int kLoadWarps = 12;                     // warps 4-15
constexpr int kMmaWarp = kEpiWarps + kLoadWarps;   // warp 16
constexpr int kUmThreads = (kMmaWarp + 1) * 32;    // 544
constexpr int kLoadThreads = kLoadWarps * 32;
constexpr int kLoadGroups = 3;                      // loader groups of 128 threads
constexpr int kStages = 4;                          // A stages in TMEM, filled in rotation
constexpr int kStageMembers = 32;                   // members per stage: one 64-real K atom
constexpr int kLoadItems = kStageMembers / 4;       // 4-member chunks per loader thread per stage
constexpr uint32_t kSuspendNs = 20000;             // hardware suspend hint per try_wait poll
constexpr uint32_t kSpinLimit = 1u << 16;          // polls before a wait gives up (<= ~1.3 s)

// error bits recorded in g_umma_error
constexpr uint32_t kErrLoaderWait = 1, kErrMmaFullWait = 2, kErrMmaAccWait = 4,
                   kErrEpilogueWait = 8, kErrDrainWait = 16, kErrProducerWait = 32,
                   kErrConvertWait = 64;

__device__ uint32_t g_umma_error;

std::atomic<int> g_tensor_loader{0};  // 0 / 1 register loaders, 2 TMA where eligible
bool tma_enabled() { return g_tensor_loader.load() == 2; }

template <int K, bool kStage> struct UmCfg {
  static constexpr int D = 1 << K;
  static constexpr int R = 2 * D;                          // reals per group: MMA N and K extent
  static constexpr int KH = D / kStageMembers;             // stages (K atoms) per tile
  static constexpr int LG = kLoadGroups;                   // loader groups
  static constexpr int GS = kLoadThreads / LG;             // threads per loader group: one per group row
  static constexpr uint32_t ATOM_G = R * 128;              // one 64-wide K block of Mr
  static constexpr uint32_t GBYTES = R * R * 2;            // one BF16 gate (hi or lo)
  static constexpr int S = kStages;
  static constexpr uint32_t ACOLS = 2 * kStageMembers;     // one A stage in TMEM: hi then lo columns
  static constexpr uint32_t COL_A = 2 * R;                 // after two FP32 accumulators of N = R columns
  static constexpr uint32_t TCOLS = 512;
  static constexpr uint32_t NBARS = 2 * S + 5;             // full, empty, accfull x2, accempty x2, drain
  static constexpr uint32_t OFF_BARS = 2 * GBYTES;
  static constexpr uint32_t OFF_MOFF = OFF_BARS + NBARS * 8;         // member offsets (u64 x D)
  static constexpr uint32_t OFF_GBASE = OFF_MOFF + D * 8;            // group bases (u64 x 128)
  static constexpr uint32_t OFF_MISC = OFF_GBASE + kTileGroups * 8;   // tmem slot, abort flag
  static constexpr uint32_t STG_ROW = 144;                            // one group's 128-byte chunk + pad
  static constexpr uint32_t OFF_STG = (OFF_MISC + 16 + 15) & ~15u;    // epilogue staging, low targets
  static constexpr uint32_t SMEM =
      OFF_STG + (kStage ? kEpiWarps * 32 * STG_ROW : 0) + 1024;  // + alignment slack
  // kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major,
  // N = R, M = 128.
  static constexpr uint32_t IDESC =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(R >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  static_assert(LG * GS == kLoadThreads && GS == kTileGroups && KH * kStageMembers == D,
                "one loader thread per group row, whole K atoms per stage");
  static_assert(K >= 5 && R % 64 == 0 && R <= 256, "N, and K blocks of one 128-byte swizzle atom");
  static_assert(COL_A + S * ACOLS <= TCOLS, "TMEM columns");
  static_assert(SMEM <= 227 * 1024, "shared memory");
  static_assert(OFF_STG % 16 == 0 && STG_ROW % 16 == 0 && OFF_GBASE % 8 == 0, "alignment");
};

struct TcTargets {
  uint64_t lo_mask[kMaxGateQubits];
  uint64_t stride[kMaxGateQubits];
};

template <int K>
__device__ __forceinline__ uint64_t tc_base(uint64_t g, const TcTargets &t) {
#pragma unroll
  for (int b = 0; b < K; ++b) g = ((g & ~t.lo_mask[b]) << 1) | (g & t.lo_mask[b]);
  return g;
}

template <int K>
__device__ __forceinline__ uint64_t tc_off(int a, const TcTargets &t) {
  uint64_t o = 0;
#pragma unroll
  for (int b = 0; b < K; ++b)
    if ((a >> b) & 1) o += t.stride[b];
  return o;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(a) : "memory");
}
// One poll: the thread is suspended in hardware until the phase completes or
// kSuspendNs elapse, so waiting warps take no issue slots from working ones.
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of parity `parity`.  Returns false when another
// role has aborted or the poll limit expired (then the abort flag and `code`
// are recorded).
__device__ __noinline__ bool mbar_wait(uint32_t a, uint32_t parity, volatile uint32_t *abort_flag,
                                       uint32_t code) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try(a, parity)) return true;
    if ((i & 15) == 15 && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicOr(&g_umma_error, code);
  return false;
}
// Warp-uniform form: lane 0 waits, the outcome is broadcast.
__device__ __forceinline__ bool mbar_wait_warp(uint32_t a, uint32_t parity,
                                               volatile uint32_t *abort_flag, uint32_t code) {
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(a, parity, abort_flag, code) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   mbar)
               : "memory");
}
// 32 lanes x 32 consecutive FP32 columns; the wait is in the same asm block so
// no use of the registers can be scheduled before the data has landed.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns from registers into tensor memory.
__device__ __forceinline__ void tc_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
      "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]),
      "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]),
      "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]),
      "r"(v[30]), "r"(v[31])
      : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns from registers into tensor memory.
__device__ __forceinline__ void tc_st16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16};\n" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
      "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}

// Shared-memory matrix descriptor, K-major with the 128-byte swizzle: rows of
// 128 bytes (64 BF16 along K), 8-row atoms 1024 bytes apart (SBO), leading
// offset unused (1), version 1 (bits 46-47), layout type 2 (bits 61-63).  The
// start address steps by 32 bytes per k16 inside an atom.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ uint32_t bf162_bits(__nv_bfloat162 v) {
  return *reinterpret_cast<uint32_t *>(&v);
}

// Off: type of the member offsets (uint32_t while every amplitude index fits,
// which makes each load/store address one wide multiply-add).
// kStage: qubit 0 is a target (members 2i, 2i+1 adjacent), so the epilogue
// stages each group's 128-byte chunk through shared memory and writes member
// pairs; the staging area exists only in this instance, since shared memory is
// carved from the same array as the L1 that holds the loads in flight.
// quad (runtime): qubits 0 and 1 are both targets, a chunk's 4 members are 32
// contiguous bytes and the loaders read them as two 16-byte vectors.
template <int K, typename Off, bool kStage>
__global__ void __launch_bounds__(kUmThreads, 1)
    k_gate_umma(float2 *__restrict__ psi, uint64_t n_groups, TcTargets t,
                const uint4 *__restrict__ gate, int quad) {
  using C = UmCfg<K, kStage>;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  const uint32_t s_gate = smem_u32(sm);               // hi at +0, lo at +GBYTES
  const uint32_t s_bar = s_gate + C::OFF_BARS;
  auto full_bar = [&](int s) { return s_bar + 8u * s; };
  auto empty_bar = [&](int s) { return s_bar + 8u * (C::S + s); };
  auto accfull_bar = [&](int b) { return s_bar + 8u * (2 * C::S + b); };
  auto accempty_bar = [&](int b) { return s_bar + 8u * (2 * C::S + 2 + b); };
  const uint32_t drain_bar = s_bar + 8u * (2 * C::S + 4);
  Off *moff = reinterpret_cast<Off *>(sm + C::OFF_MOFF);
  uint64_t *gbase = reinterpret_cast<uint64_t *>(sm + C::OFF_GBASE);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + C::OFF_MISC);
  volatile uint32_t *abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t n_tiles = (n_groups + kTileGroups - 1) / kTileGroups;

  // gate (packed on the host in the operand layout) and member offsets
  {
    uint4 *dst = reinterpret_cast<uint4 *>(sm);
    for (uint32_t i = threadIdx.x; i < 2 * C::GBYTES / 16; i += kUmThreads) dst[i] = gate[i];
    for (int m = threadIdx.x; m < C::D; m += kUmThreads) moff[m] = (Off)tc_off<K>(m, t);
    for (int g = threadIdx.x; g < kTileGroups; g += kUmThreads) gbase[g] = tc_base<K>((uint64_t)g, t);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::S; ++s) {
      mbar_init(full_bar(s), C::GS);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accfull_bar(b), 1);
      mbar_init(accempty_bar(b), kEpiWarps * 32);
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  fence_async_smem();  // the gate's generic stores become visible to the tensor core
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(C::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kMmaWarp) {
    // ---- MMA issuer ----------------------------------------------------------
    // tile `it` consumes stages h = it * KH .. it * KH + KH - 1 (one K atom each)
    uint32_t it = 0;
    bool issued = false, ok = true;
    for (uint64_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x, ++it) {
      const uint32_t b = it & 1, v = it >> 1;
      for (int kp = 0; kp < C::KH; ++kp) {
        const uint32_t h = it * C::KH + kp, s = h % C::S, u = h / C::S;
        if (!mbar_wait_warp(full_bar(s), u & 1, abort_flag, kErrMmaFullWait)) { ok = false; break; }
        if (kp == 0 && !mbar_wait_warp(accempty_bar(b), (v & 1) ^ 1, abort_flag, kErrMmaAccWait)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t gh = s_gate + kp * C::ATOM_G, gl = gh + C::GBYTES;
          const uint32_t d = tmem + b * C::R;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            // K reals kp * 64 + ks * 16 .. +15: 8 columns of the stage's hi and lo blocks
            const uint32_t ah = tmem + C::COL_A + s * C::ACOLS + ks * 8, al = ah + kStageMembers;
            const uint64_t b_hi = umma_desc_sw128(gh + ks * 32), b_lo = umma_desc_sw128(gl + ks * 32);
            tc_mma_ts(d, al, b_hi, C::IDESC, (kp > 0 || ks > 0) ? 1u : 0u);
            tc_mma_ts(d, ah, b_lo, C::IDESC, 1u);
            tc_mma_ts(d, ah, b_hi, C::IDESC, 1u);
          }
          tc_commit(empty_bar(s));
          if (kp == C::KH - 1) tc_commit(accfull_bar(b));
        }
        __syncwarp();
        issued = true;
      }
    }
    // every MMA of this CTA has completed before tensor memory is released
    if (issued) {
      if (lane == 0) tc_commit(drain_bar);
      __syncwarp();
      volatile uint32_t never = 0;
      mbar_wait_warp(drain_bar, 0, &never, kErrDrainWait);
    }
  } else if (warp >= kEpiWarps) {
    // ---- loaders: HBM -> split BF16 -> operand stage --------------------------
    // thread (lg, gg) loads group row gg of the stages group lg owns: 32 members
    // (8 chunks of 4) per stage, so a warp instruction covers 32 consecutive
    // groups of one member.
    const int lt = threadIdx.x - kEpiWarps * 32;
    const int lg = lt / C::GS, gg = lt % C::GS;  // group row gg of every tile
    const uint64_t gb = tc_base<K>((uint64_t)gg, t);
    // the A stages' columns in this warp's TMEM sub-partition (lanes of groups gg & ~31)
    const uint32_t acol0 = tmem + ((uint32_t)(gg & ~31) << 16) + C::COL_A;
    // stage h holds K atom h % KH of tile h / KH in slot h % S; group lg fills
    // stages h = lg, lg + LG, ...  Before it waits for slot h % S to be free
    // (stage h - S consumed), it has seen stage h - LG - S consumed, so the wait
    // is never more than one phase ahead of the slot's barrier.
    for (uint32_t h = lg;; h += C::LG) {
      const uint32_t ti = h / C::KH, kp = h % C::KH, u = h / C::S, sl = h % C::S;
      const uint32_t acol = acol0 + sl * C::ACOLS;
      const uint64_t tile = blockIdx.x + (uint64_t)ti * gridDim.x;
      if (tile >= n_tiles) break;
      const bool live = tile * kTileGroups + gg < n_groups;
      const float2 *p = psi + tc_base<K>(tile * kTileGroups, t) + gb;
      float2 v[kLoadItems][4];
#pragma unroll
      for (int j = 0; j < kLoadItems; ++j) {
        const int c = kp * kLoadItems + j;
        if (live) {
          if (kStage && quad) {
            const float4 a = *reinterpret_cast<const float4 *>(p + moff[4 * c]);
            const float4 b = *reinterpret_cast<const float4 *>(p + moff[4 * c] + 2);
            v[j][0] = make_float2(a.x, a.y);
            v[j][1] = make_float2(a.z, a.w);
            v[j][2] = make_float2(b.x, b.y);
            v[j][3] = make_float2(b.z, b.w);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) v[j][q] = p[moff[4 * c + q]];
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) v[j][q] = make_float2(0.f, 0.f);
        }
      }
      if (!mbar_wait_warp(empty_bar(sl), (u & 1) ^ 1, abort_flag, kErrLoaderWait)) break;
      tc_fence_after();
      // member 4 j + q of the stage is column 4 j + q of the hi and of the lo block
      uint32_t hb[kStageMembers], lb[kStageMembers];
#pragma unroll
      for (int j = 0; j < kLoadItems; ++j) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __nv_bfloat162 hv = __floats2bfloat162_rn(v[j][q].x, v[j][q].y);
          const uint32_t h2 = bf162_bits(hv);
          hb[4 * j + q] = h2;
          lb[4 * j + q] = bf162_bits(__floats2bfloat162_rn(v[j][q].x - __uint_as_float(h2 << 16),
                                                           v[j][q].y - __uint_as_float(h2 & 0xFFFF0000u)));
        }
      }
      tc_st32(acol, hb);
      tc_st32(acol + kStageMembers, lb);
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      tc_fence_before();
      mbar_arrive(full_bar(sl));
    }
  } else {
    // ---- epilogue: TMEM -> registers -> HBM -----------------------------------
    const int gg = warp * 32 + lane;
    const uint64_t gb = tc_base<K>((uint64_t)gg, t);
    unsigned char *stg = sm + C::OFF_STG + warp * 32 * C::STG_ROW;
    uint32_t it = 0;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++it) {
      const uint32_t b = it & 1, v = it >> 1;
      if (!mbar_wait_warp(accfull_bar(b), v & 1, abort_flag, kErrEpilogueWait)) break;
      tc_fence_after();
      const bool live = tile * kTileGroups + gg < n_groups;
      float2 *const tb = psi + tc_base<K>(tile * kTileGroups, t);
      float2 *p = tb + gb;
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + b * C::R;
#pragma unroll
      for (int cc = 0; cc < C::R / 32; ++cc) {
        float r[32];
        tc_ld32(taddr + cc * 32, r);
        if (cc == C::R / 32 - 1) {
          tc_fence_before();
          mbar_arrive(accempty_bar(b));
        }
        if constexpr (!kStage) {
          // qubit 0 is not a target: groups gg and gg ^ 1 are adjacent amplitudes, so
          // lane pairs swap one member and each writes a 16-byte (even, odd group)
          // pair: half the store instructions, and whole sectors when the warp's
          // groups are not one contiguous run (targets 1..6: 4.96 -> 3.69 ms at 30
          // qubits).  Both groups of a pair are live or neither (n_groups is even).
          const bool odd = lane & 1;
          float2 *pe = odd ? p - 1 : p;  // the even group's address
#pragma unroll
          for (int j = 0; j < 16; j += 2) {
            const float2 mine0 = make_float2(r[2 * j], r[2 * j + 1]);
            const float2 mine1 = make_float2(r[2 * j + 2], r[2 * j + 3]);
            const float2 give = odd ? mine0 : mine1;
            float2 got;
            got.x = __shfl_xor_sync(0xffffffffu, give.x, 1);
            got.y = __shfl_xor_sync(0xffffffffu, give.y, 1);
            const float4 v = odd ? make_float4(got.x, got.y, mine1.x, mine1.y)
                                 : make_float4(mine0.x, mine0.y, got.x, got.y);
            if (live) *reinterpret_cast<float4 *>(pe + moff[cc * 16 + j + (odd ? 1 : 0)]) = v;
          }
        } else {
          // a group's 16 members of this chunk go to its staging row; then the
          // warp writes member pairs (16 bytes), 4 groups x 8 pairs per instruction
          unsigned char *row = stg + lane * C::STG_ROW;
#pragma unroll
          for (int j = 0; j < 8; ++j)
            *reinterpret_cast<float4 *>(row + 16 * j) =
                make_float4(r[4 * j], r[4 * j + 1], r[4 * j + 2], r[4 * j + 3]);
          __syncwarp();
          const int pj = lane & 7;
#pragma unroll
          for (int rd = 0; rd < 8; ++rd) {
            const int gi = rd * 4 + (lane >> 3), g2 = warp * 32 + gi;
            const float4 val = *reinterpret_cast<const float4 *>(stg + gi * C::STG_ROW + 16 * pj);
            if (tile * kTileGroups + g2 < n_groups)
              *reinterpret_cast<float4 *>(tb + gbase[g2] + moff[cc * 16 + 2 * pj]) = val;
          }
          __syncwarp();
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(C::TCOLS)
                 : "memory");
  }
}

// ---- TMA-fed variant (loader mode 2) -------------------------------------------
// For gates whose lowest target qubit is >= 7 (launched for those only; the kernel
// itself handles runs of 2^min(q0, 7) amplitudes), the 128 groups of a tile are
// one contiguous 1 KB run for every member, so the raw FP32 tile can be fetched
// with TMA bulk copies (cp.async.bulk, completion counted on an mbarrier) into
// a ring of raw slots, one 32-member K atom per slot; the copies occupy neither
// L1 nor registers.  Warps:
//   0-7   epilogue: warp w reads TMEM sub-partition w % 4 (32 groups) and half
//         w / 4 of the accumulator columns;
//   8-15  converters: thread (gg, half) splits members 16 half .. 16 half + 15
//         of group row gg of a raw slot into the A stage in tensor memory;
//   16    producer: lane 0 arms the slot's mbarrier with the slot's bytes, the 32
//         lanes issue its bulk copies; before exiting it waits (bounded) for the
//         copies of the last slots it armed;
//   17    TMEM allocation and MMA issue, as in k_gate_umma.
constexpr int kTEpiWarps = 8;                         // two per TMEM sub-partition
constexpr int kTConvWarps = 8;
constexpr int kTProdWarp = kTEpiWarps + kTConvWarps;  // 16
constexpr int kTMmaWarp = kTProdWarp + 1;             // 17
constexpr int kTThreads = (kTMmaWarp + 1) * 32;       // 576
constexpr int kTConvThreads = kTConvWarps * 32;

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t smem_dst, const void *gmem_src, uint32_t bytes,
                                         uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_dst),
      "l"(gmem_src), "r"(bytes), "r"(mbar)
      : "memory");
}

// The data operand sits in tensor memory as in k_gate_umma, so the 64 KB gate
// leaves room for five 32 KB raw slots (160 KB of copies in flight per SM).
// Tensor memory: accumulators at columns 0 and R, four A stages of 64 columns
// from 2R (512 columns).  Converter warp w writes lanes 32 (w % 4) .. +31, the
// groups it converts.
template <int K> struct UxCfg {
  static constexpr int D = 1 << K;
  static constexpr int R = 2 * D;
  static constexpr int KH = D / kStageMembers;             // K atoms (slots, A stages) per tile
  static constexpr int S = 4;                              // A stages in tensor memory
  static constexpr int RS = 5;                             // raw slots
  static constexpr uint32_t ATOM_G = R * 128;
  static constexpr uint32_t RAW = kStageMembers * kTileGroups * 8;
  static constexpr uint32_t GBYTES = R * R * 2;
  static constexpr uint32_t ACOLS = 2 * kStageMembers;     // hi then lo, one column a member
  static constexpr uint32_t COL_A = 2 * R;
  static constexpr uint32_t TCOLS = 512;
  static constexpr uint32_t NBARS = 2 * RS + 2 * S + 5;
  static constexpr uint32_t OFF_RAW = 2 * GBYTES;
  static constexpr uint32_t OFF_BARS = OFF_RAW + RS * RAW;
  static constexpr uint32_t OFF_MOFF = OFF_BARS + NBARS * 8;
  static constexpr uint32_t OFF_GBASE = OFF_MOFF + D * 8;
  static constexpr uint32_t OFF_MISC = OFF_GBASE + kTileGroups * 8;
  static constexpr uint32_t SMEM = OFF_MISC + 16 + 1024;
  static constexpr uint32_t IDESC =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(R >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  static_assert(K == 6 && KH * kStageMembers == D, "the 6-qubit gate, whole K atoms");
  static_assert(COL_A + S * ACOLS <= TCOLS, "tensor memory columns");
  static_assert(SMEM <= 227 * 1024, "shared memory");
  static_assert(OFF_RAW % 1024 == 0 && OFF_GBASE % 8 == 0, "alignment");
};

template <int K, typename Off>
__global__ void __launch_bounds__(kTThreads, 1)
    k_gate_umma_tx(float2 *__restrict__ psi, uint64_t n_groups, TcTargets t,
                   const uint4 *__restrict__ gate, int run_log2) {
  using C = UxCfg<K>;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char *sm = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  const uint32_t s_gate = smem_u32(sm);
  const uint32_t s_bar = s_gate + C::OFF_BARS;
  auto raw_full = [&](int r) { return s_bar + 8u * r; };
  auto raw_empty = [&](int r) { return s_bar + 8u * (C::RS + r); };
  auto a_full = [&](int q) { return s_bar + 8u * (2 * C::RS + q); };
  auto a_empty = [&](int q) { return s_bar + 8u * (2 * C::RS + C::S + q); };
  auto accfull_bar = [&](int b) { return s_bar + 8u * (2 * C::RS + 2 * C::S + b); };
  auto accempty_bar = [&](int b) { return s_bar + 8u * (2 * C::RS + 2 * C::S + 2 + b); };
  const uint32_t drain_bar = s_bar + 8u * (2 * C::RS + 2 * C::S + 4);
  Off *moff = reinterpret_cast<Off *>(sm + C::OFF_MOFF);
  uint64_t *gbase = reinterpret_cast<uint64_t *>(sm + C::OFF_GBASE);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + C::OFF_MISC);
  volatile uint32_t *abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t n_tiles = n_groups / kTileGroups;  // whole tiles only (checked on the host)

  {
    uint4 *dst = reinterpret_cast<uint4 *>(sm);
    for (uint32_t i = threadIdx.x; i < 2 * C::GBYTES / 16; i += kTThreads) dst[i] = gate[i];
    for (int m = threadIdx.x; m < C::D; m += kTThreads) moff[m] = (Off)tc_off<K>(m, t);
    for (int g = threadIdx.x; g < kTileGroups; g += kTThreads) gbase[g] = tc_base<K>((uint64_t)g, t);
  }
  if (threadIdx.x == 0) {
    for (int r = 0; r < C::RS; ++r) {
      mbar_init(raw_full(r), 1);
      mbar_init(raw_empty(r), kTConvThreads);
    }
    for (int q = 0; q < C::S; ++q) {
      mbar_init(a_full(q), kTConvThreads);
      mbar_init(a_empty(q), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accfull_bar(b), 1);
      mbar_init(accempty_bar(b), kTEpiWarps * 32);
    }
    mbar_init(drain_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  fence_async_smem();
  if (warp == kTMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(C::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kTMmaWarp) {
    // ---- MMA issuer: tile `it` consumes A stages h = it * KH + kp --------------
    uint32_t it = 0;
    bool issued = false, ok = true;
    for (uint64_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x, ++it) {
      const uint32_t b = it & 1, v = it >> 1;
      for (int kp = 0; kp < C::KH; ++kp) {
        const uint32_t h = it * C::KH + kp, q = h % C::S, u = h / C::S;
        if (!mbar_wait_warp(a_full(q), u & 1, abort_flag, kErrMmaFullWait)) { ok = false; break; }
        if (kp == 0 && !mbar_wait_warp(accempty_bar(b), (v & 1) ^ 1, abort_flag, kErrMmaAccWait)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t gh = s_gate + kp * C::ATOM_G, gl = gh + C::GBYTES;
          const uint32_t d = tmem + b * C::R;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            // K reals kp * 64 + ks * 16 .. +15: 8 columns of the stage's hi and lo blocks
            const uint32_t ah = tmem + C::COL_A + q * C::ACOLS + ks * 8, al = ah + kStageMembers;
            const uint64_t b_hi = umma_desc_sw128(gh + ks * 32), b_lo = umma_desc_sw128(gl + ks * 32);
            tc_mma_ts(d, al, b_hi, C::IDESC, (kp > 0 || ks > 0) ? 1u : 0u);
            tc_mma_ts(d, ah, b_lo, C::IDESC, 1u);
            tc_mma_ts(d, ah, b_hi, C::IDESC, 1u);
          }
          tc_commit(a_empty(q));
          if (kp == C::KH - 1) tc_commit(accfull_bar(b));
        }
        __syncwarp();
        issued = true;
      }
    }
    if (issued) {
      if (lane == 0) tc_commit(drain_bar);
      __syncwarp();
      volatile uint32_t never = 0;
      mbar_wait_warp(drain_bar, 0, &never, kErrDrainWait);
    }
  } else if (warp == kTProdWarp) {
    // ---- producer: bulk copies of raw slot h = it * KH + kp --------------------
    const int run = 1 << run_log2, runs = kTileGroups >> run_log2;
    const int copies = kStageMembers * runs;
    uint32_t h = 0;
    bool ok = true;
    for (uint64_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x) {
      const float2 *tp = psi + tc_base<K>(tile * kTileGroups, t);
      for (int kp = 0; kp < C::KH; ++kp) {
        const uint32_t r = h % C::RS, u = h / C::RS;
        if (!mbar_wait_warp(raw_empty(r), (u & 1) ^ 1, abort_flag, kErrProducerWait)) {
          ok = false;
          break;
        }
        if (lane == 0) mbar_arrive_expect_tx(raw_full(r), C::RAW);
        __syncwarp();
        const uint32_t dst0 = s_gate + C::OFF_RAW + r * C::RAW;
        for (int c = lane; c < copies; c += 32) {
          const int ml = c / runs, rr = c % runs;
          bulk_g2s(dst0 + ml * (kTileGroups * 8) + (rr << run_log2) * 8,
                   tp + gbase[rr << run_log2] + moff[kp * kStageMembers + ml], run * 8, raw_full(r));
        }
        ++h;
      }
    }
    // every copy this CTA issued has landed before its shared memory is released
    volatile uint32_t never = 0;
    for (uint32_t j = h > (uint32_t)C::RS ? h - C::RS : 0; j < h; ++j)
      mbar_wait_warp(raw_full(j % C::RS), (j / C::RS) & 1, &never, kErrDrainWait);
  } else if (warp >= kTEpiWarps) {
    // ---- converters: raw slot -> split BF16 -> A stage in tensor memory --------
    const int ct = threadIdx.x - kTEpiWarps * 32;
    const int gg = ct % kTileGroups, half = ct / kTileGroups;
    const uint32_t lanes = (uint32_t)(gg & ~31) << 16;  // this warp's TMEM sub-partition
    for (uint32_t h = 0;; ++h) {
      const uint64_t tile = blockIdx.x + (uint64_t)(h / C::KH) * gridDim.x;
      if (tile >= n_tiles) break;
      const uint32_t r = h % C::RS, ur = h / C::RS, q = h % C::S, uq = h / C::S;
      if (!mbar_wait_warp(raw_full(r), ur & 1, abort_flag, kErrConvertWait)) break;
      if (!mbar_wait_warp(a_empty(q), (uq & 1) ^ 1, abort_flag, kErrConvertWait)) break;
      tc_fence_after();
      const unsigned char *raw = sm + C::OFF_RAW + r * C::RAW + gg * 8;
      uint32_t hb[16], lb[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float2 v =
            *reinterpret_cast<const float2 *>(raw + (16 * half + i) * (kTileGroups * 8));
        const __nv_bfloat162 hv = __floats2bfloat162_rn(v.x, v.y);
        hb[i] = bf162_bits(hv);
        lb[i] = bf162_bits(__floats2bfloat162_rn(v.x - __uint_as_float(hb[i] << 16),
                                                  v.y - __uint_as_float(hb[i] & 0xFFFF0000u)));
      }
      const uint32_t col = tmem + lanes + C::COL_A + q * C::ACOLS + 16 * half;
      tc_st16(col, hb);
      tc_st16(col + kStageMembers, lb);
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      tc_fence_before();
      mbar_arrive(a_full(q));
      mbar_arrive(raw_empty(r));
    }
  } else {
    // ---- epilogue: TMEM -> registers -> HBM (qubit 0 is never a target here) ----
    const int quarter = warp & 3, half = warp >> 2;
    const int gg = quarter * 32 + lane;
    const uint64_t gb = gbase[gg];
    constexpr int CPW = C::R / 64;  // 32-column chunks per epilogue warp
    uint32_t it = 0;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++it) {
      const uint32_t b = it & 1, v = it >> 1;
      if (!mbar_wait_warp(accfull_bar(b), v & 1, abort_flag, kErrEpilogueWait)) break;
      tc_fence_after();
      float2 *p = psi + tc_base<K>(tile * kTileGroups, t) + gb;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + b * C::R + half * CPW * 32;
#pragma unroll
      for (int ci = 0; ci < CPW; ++ci) {
        const int cc = half * CPW + ci;
        float rr[32];
        tc_ld32(taddr + ci * 32, rr);
        if (ci == CPW - 1) {
          tc_fence_before();
          mbar_arrive(accempty_bar(b));
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) p[moff[cc * 16 + j]] = make_float2(rr[2 * j], rr[2 * j + 1]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(C::TCOLS)
                 : "memory");
  }
}

uint16_t bf16_bits_rn(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

float bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

template <int K, typename Off, bool kStage>
bool launch_um_k(const uint32_t *qubits, const void *d_tc, void *sv, uint32_t n, cudaStream_t s,
                 std::string &err) {
  using C = UmCfg<K, kStage>;
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  static int blocks_per_sm = 1;
  std::call_once(once, [] {
    attr_rc = cudaFuncSetAttribute(k_gate_umma<K, Off, kStage>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)C::SMEM);
    int b = 0;
    if (attr_rc == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_gate_umma<K, Off, kStage>, kUmThreads, C::SMEM) ==
            cudaSuccess &&
        b > 0)
      blocks_per_sm = std::min(b, (int)(512 / C::TCOLS));
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(tensor gate kernel)", err)) return false;
  TcTargets t;
  for (uint32_t b = 0; b < kMaxGateQubits; ++b) {
    const uint32_t q = b < (uint32_t)K ? qubits[b] : 0;
    t.lo_mask[b] = (1ull << q) - 1;
    t.stride[b] = 1ull << q;
  }
  const uint64_t n_groups = 1ull << (n - K);
  const uint64_t n_tiles = (n_groups + kTileGroups - 1) / kTileGroups;
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(n_tiles, (uint64_t)blocks_per_sm * sm_count()));
  const int quad = kStage && qubits[1] == 1;
  k_gate_umma<K, Off, kStage><<<grid, kUmThreads, C::SMEM, s>>>(
      static_cast<float2 *>(sv), n_groups, t, static_cast<const uint4 *>(d_tc), quad);
  return cuda_ok(cudaGetLastError(), "tensor gate kernel launch", err);
}

template <int K, typename Off>
bool launch_ux_k(const uint32_t *qubits, const void *d_tc, void *sv, uint32_t n, cudaStream_t s,
                 std::string &err) {
  using C = UxCfg<K>;
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  std::call_once(once, [] {
    attr_rc = cudaFuncSetAttribute(k_gate_umma_tx<K, Off>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)C::SMEM);
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(tensor gate kernel, TMA, A in TMEM)", err)) return false;
  TcTargets t;
  for (uint32_t b = 0; b < kMaxGateQubits; ++b) {
    const uint32_t q = b < (uint32_t)K ? qubits[b] : 0;
    t.lo_mask[b] = (1ull << q) - 1;
    t.stride[b] = 1ull << q;
  }
  const uint64_t n_tiles = (1ull << (n - K)) / kTileGroups;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(n_tiles, (uint64_t)sm_count()));
  const int run_log2 = (int)std::min<uint32_t>(qubits[0], 7);
  k_gate_umma_tx<K, Off><<<grid, kTThreads, C::SMEM, s>>>(
      static_cast<float2 *>(sv), 1ull << (n - K), t, static_cast<const uint4 *>(d_tc), run_log2);
  return cuda_ok(cudaGetLastError(), "tensor gate kernel launch (TMA, A in TMEM)", err);
}

}  // namespace

bool tensor_path_supported(const GateData &g) {
  return g.precision == 0 && g.k >= 5 && g.k <= 6;
}

// Packs Mr (R x R, Mr[2r+c'][2m+c] as in the header) as the MMA's K-major
// operand with the 128-byte swizzle: element (row, col) at byte
// (col / 64) * R * 128 + row * 128 + (((col % 64) / 8 ^ row % 8) * 16) + (col % 8) * 2;
// hi block first, then lo.  m64 is the D x D matrix, interleaved re/im.
std::vector<uint16_t> pack_tensor_operand(const double *m64, int k) {
  const int D = 1 << k, R = 2 * D;
  const size_t per = (size_t)R * R;
  std::vector<uint16_t> packed(2 * per);
  for (int row = 0; row < R; ++row)
    for (int col = 0; col < R; ++col) {
      const int r = row >> 1, m = col >> 1;
      const double a = m64[2 * ((size_t)r * D + m)], b = m64[2 * ((size_t)r * D + m) + 1];
      const bool out_im = row & 1, in_im = col & 1;
      const double v = out_im ? (in_im ? a : b) : (in_im ? -b : a);
      const uint16_t hi = bf16_bits_rn((float)v);
      const uint16_t lo = bf16_bits_rn((float)(v - (double)bf16_value(hi)));
      const size_t byte = (size_t)(col / 64) * R * 128 + (size_t)row * 128 +
                          ((size_t)(((col % 64) / 8) ^ (row % 8)) << 4) + (col % 8) * 2;
      packed[byte / 2] = hi;
      packed[per + byte / 2] = lo;
    }
  return packed;
}

// A 5-qubit gate runs on the 6-qubit kernel, padded with the identity on a spare
// qubit: the tensor pass is bound by memory, not by the tensor pipe, and the
// 6-qubit tile moves twice the bytes per tile handoff (measured at 30 qubits:
// 4.3 ms for a 5-qubit pass, 3.6 ms for a 6-qubit one).  The spare qubit is the
// lowest non-target >= 7 when there is one (a gate whose targets are all >= 7
// stays eligible for the bulk-copy loaders), else the highest non-target.
bool prepare_tensor_gate(GateData &g, uint32_t n, std::string &err) {
  if (!tensor_path_supported(g)) {
    err = "the tensor-core path takes complex64 gates with 5 or 6 qubits";
    return false;
  }
  std::vector<uint16_t> packed;
  g.tc_k = g.k;
  for (uint32_t b = 0; b < g.k; ++b) g.tc_qubits[b] = g.qubits[b];
  if (g.k == 5 && n > 5) {
    uint32_t used = 0;
    for (uint32_t b = 0; b < 5; ++b) used |= 1u << g.qubits[b];
    int spare = -1;
    for (uint32_t c = 7; c < n && spare < 0; ++c)
      if (!((used >> c) & 1)) spare = (int)c;
    for (int c = (int)n - 1; c >= 0 && spare < 0; --c)
      if (!((used >> c) & 1)) spare = c;
    uint32_t q6[6], j = 0, pos = 0;
    for (uint32_t b = 0, i = 0; b < 6; ++b) {
      if (j == 0 && (i == 5 || (uint32_t)spare < g.qubits[i])) {
        q6[b] = (uint32_t)spare;
        pos = b;
        j = 1;
      } else {
        q6[b] = g.qubits[i++];
      }
    }
    // M6[r][c] = M5[r without bit pos][c without bit pos] when bit pos of r and c agree, else 0
    std::vector<double> m6(2 * 64 * 64, 0.0);
    auto drop = [&](uint32_t x) { return ((x >> (pos + 1)) << pos) | (x & ((1u << pos) - 1)); };
    for (uint32_t r = 0; r < 64; ++r)
      for (uint32_t c = 0; c < 64; ++c)
        if (((r >> pos) & 1) == ((c >> pos) & 1)) {
          const size_t src = 2 * ((size_t)drop(r) * 32 + drop(c)), dst = 2 * ((size_t)r * 64 + c);
          m6[dst] = g.m64[src];
          m6[dst + 1] = g.m64[src + 1];
        }
    packed = pack_tensor_operand(m6.data(), 6);
    g.tc_k = 6;
    for (uint32_t b = 0; b < 6; ++b) g.tc_qubits[b] = q6[b];
  } else {
    packed = pack_tensor_operand(g.m64.data(), (int)g.k);
  }
  if (g.d_tc) cudaFree(g.d_tc);
  g.d_tc = nullptr;
  if (!cuda_ok(cudaMalloc(&g.d_tc, packed.size() * 2), "cudaMalloc (tensor gate operand)", err))
    return false;
  return cuda_ok(cudaMemcpy(g.d_tc, packed.data(), packed.size() * 2, cudaMemcpyHostToDevice),
                 "cudaMemcpy (tensor gate operand)", err);
}

bool launch_gate_tensor(const GateData &g, void *sv, uint32_t n, cudaStream_t s, std::string &err) {
  if (!g.d_tc || !tensor_path_supported(g) || (g.tc_k != 5 && g.tc_k != 6) || n < g.tc_k) {
    err = "gate has no tensor-core operand for this statevector";
    return false;
  }
  const uint32_t *q = g.tc_qubits;
  const void *op = g.d_tc;
  // member offsets are below 2^n amplitudes: 32-bit while n <= 32
  const bool narrow = n <= 32, stage = q[0] == 0;
  // TMA bulk-copy feed on request only (loader mode 2), for a lowest target >= 7
  // and whole tiles, where every member's 128 groups are one 1 KB run: with the
  // data operand in tensor memory the register loaders measured faster (one
  // 30-qubit 6-qubit gate, high targets: 2.82 ms against 3.04 ms)
  if (g.tc_k == 6 && q[0] >= 7 && n >= 6 + 7 && tma_enabled())
    return narrow ? launch_ux_k<6, uint32_t>(q, op, sv, n, s, err)
                  : launch_ux_k<6, uint64_t>(q, op, sv, n, s, err);
  if (g.tc_k == 5) {
    if (narrow) return stage ? launch_um_k<5, uint32_t, true>(q, op, sv, n, s, err)
                             : launch_um_k<5, uint32_t, false>(q, op, sv, n, s, err);
    return stage ? launch_um_k<5, uint64_t, true>(q, op, sv, n, s, err)
                 : launch_um_k<5, uint64_t, false>(q, op, sv, n, s, err);
  }
  if (narrow) return stage ? launch_um_k<6, uint32_t, true>(q, op, sv, n, s, err)
                           : launch_um_k<6, uint32_t, false>(q, op, sv, n, s, err);
  return stage ? launch_um_k<6, uint64_t, true>(q, op, sv, n, s, err)
               : launch_um_k<6, uint64_t, false>(q, op, sv, n, s, err);
}

int set_tensor_loader(int mode) { return g_tensor_loader.exchange(mode); }

// Reads and clears the tensor kernel's error word (a bit per wait that expired).
bool tensor_error_status(uint32_t *out, std::string &err) {
  uint32_t zero = 0;
  // launches on non-blocking streams are not ordered with the legacy stream's copy
  if (!cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize (tensor error word)", err)) return false;
  if (!cuda_ok(cudaMemcpyFromSymbol(out, g_umma_error, sizeof(uint32_t)),
               "cudaMemcpyFromSymbol (tensor error word)", err))
    return false;
  return cuda_ok(cudaMemcpyToSymbol(g_umma_error, &zero, sizeof(uint32_t)),
                 "cudaMemcpyToSymbol (tensor error word)", err);
}

}  // namespace cb2

