// Tensor-core gate application for complex64 statevectors, k = 4, 5, 6.
//
// A fused k-qubit gate M = A + iB (2^k x 2^k) applied to G gather groups is the
// real GEMM
//     [Yr]   [A  -B] [Xr]
//     [Yi] = [B   A] [Xi]        (R x R) x (R x G),  R = 2^(k+1),
// with one column per group (X rows = real parts then imaginary parts of the
// group's 2^k members).  It runs on the tensor cores in split BF16: every FP32
// operand v is written as hi + lo with hi = bf16(v), lo = bf16(v - hi), and
// Y = A_lo X_hi + A_hi X_lo + A_hi X_hi with FP32 accumulation (the lo*lo term,
// below 2^-16 of the product, is dropped).  Relative error per product is about
// 2^-16, so a fused pass changes an amplitude by ~1e-5 of the norm of its group
// - the bound the tests state.
//
// Kernel: persistent CTAs of 8 warps; each warp keeps its 16-row slices of
// A_hi / A_lo as mma.sync A fragments in registers (packed on the host in
// fragment order) for the whole launch.  Tiles of 64 groups (64 x 2^k
// amplitudes) are fetched with cp.async into a double buffer one tile ahead
// (consecutive groups are consecutive amplitudes when the targets are high, so
// the copies coalesce), split into BF16 hi/lo in shared memory in the loaded,
// member-major orientation (rows padded by 16 bytes), turned into B fragments
// by ldmatrix.trans and multiplied with m16n8k16 BF16 MMAs; the FP32 result is
// staged through the same shared memory and stored back coalesced (stores
// straight from the accumulator fragments scatter over 8 member rows per
// instruction and measured slower).
#include "internal.hpp"

#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

namespace cb2 {

namespace {

constexpr int kTcThreads = 256;
constexpr int kTcG = 64;  // groups per tile

template <int K> struct TcCfg {
  static constexpr int D = 1 << K;
  static constexpr int R = 2 * D;             // real rows / columns of the GEMM
  static constexpr int MT = R / 16;           // m16 tiles
  static constexpr int WN = 8 / MT;           // warps sharing one m-tile
  static constexpr int NF = (kTcG / 8) / WN;  // n8 fragments per warp
  static constexpr int KS = R / 16;           // k16 steps
  static constexpr int SN = kTcG + 8;         // bf16 elements per X row (one row per real input)
  static constexpr int AMPS = kTcG * D;        // amplitudes per tile
  static constexpr int PER = AMPS / kTcThreads;  // per thread
  static constexpr size_t STAGE = 2ull * AMPS * sizeof(float2);  // double-buffered raw tiles
  static constexpr int SG = kTcG + 4;         // floats per staged result row
  static constexpr size_t XBYTES = 2ull * R * SN * sizeof(__nv_bfloat16);
  static constexpr size_t YBYTES = (size_t)R * SG * sizeof(float);
  static constexpr size_t SMEM = STAGE + (XBYTES > YBYTES ? XBYTES : YBYTES);
};

__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gmem_src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
// Four transposed 8x8 b16 tiles: lanes 8j..8j+7 give the row addresses of tile j.
__device__ __forceinline__ void ldsm_x4_trans(uint32_t (&r)[4], const void *row_addr) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(row_addr);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

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

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The raw tile of the next iteration is fetched with cp.async into the other
// half of a double buffer while this iteration splits, multiplies and stores.
template <int K>
__global__ void __launch_bounds__(kTcThreads, 2)
    k_gate_tc(float2 *__restrict__ psi, uint64_t n_groups, TcTargets t,
              const uint32_t *__restrict__ afrag) {
  using C = TcCfg<K>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2 *stage = reinterpret_cast<float2 *>(smem_raw);  // [2][D][kTcG]
  unsigned char *xy = smem_raw + C::STAGE;
  __nv_bfloat16 *Xhi = reinterpret_cast<__nv_bfloat16 *>(xy);
  __nv_bfloat16 *Xlo = Xhi + C::R * C::SN;
  float *Ys = reinterpret_cast<float *>(xy);  // aliases X once the MMAs are done
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = warp % C::MT, wn = warp / C::MT;
  uint32_t ah[C::KS][4], al[C::KS][4];
  const uint32_t *fh = afrag, *fl = afrag + (size_t)C::MT * C::KS * 128;
#pragma unroll
  for (int ks = 0; ks < C::KS; ++ks)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const size_t idx = (((size_t)mt * C::KS + ks) * 32 + lane) * 4 + i;
      ah[ks][i] = fh[idx];
      al[ks][i] = fl[idx];
    }
  const uint64_t n_tiles = (n_groups + kTcG - 1) / kTcG;
  auto issue = [&](uint64_t tile, int buf) {
    const uint64_t g0 = tile * kTcG;
    float2 *dst = stage + buf * C::AMPS;
#pragma unroll
    for (int j = 0; j < C::PER; ++j) {
      const int i = threadIdx.x + j * kTcThreads;
      const int gg = i % kTcG, a = i / kTcG;
      const uint64_t g = g0 + gg;
      if (g < n_groups) cp_async8(dst + i, psi + tc_base<K>(g, t) + tc_off<K>(a, t));
      else dst[i] = make_float2(0.f, 0.f);
    }
    cp_async_commit();
  };
  uint64_t tile = blockIdx.x;
  int buf = 0;
  if (tile < n_tiles) issue(tile, 0);
  for (; tile < n_tiles; tile += gridDim.x, buf ^= 1) {
    const uint64_t next = tile + gridDim.x;
    if (next < n_tiles) issue(next, buf ^ 1);
    else cp_async_commit();  // an empty group keeps wait_group<1> meaning "tile landed"
    cp_async_wait<1>();
    __syncthreads();
    // split: member-major X[k][group]; each thread converts two adjacent groups
    // of one member (a 16-byte read, 32-bit stores, both conflict-free)
    const float2 *cur = stage + buf * C::AMPS;
#pragma unroll
    for (int j = 0; j < C::PER / 2; ++j) {
      const int i = threadIdx.x + j * kTcThreads;
      const int gg = 2 * (i % (kTcG / 2)), a = i / (kTcG / 2);
      const float4 v = *reinterpret_cast<const float4 *>(cur + a * kTcG + gg);
      const __nv_bfloat162 hr = __floats2bfloat162_rn(v.x, v.z);
      const __nv_bfloat162 hi = __floats2bfloat162_rn(v.y, v.w);
      const __nv_bfloat162 lr = __floats2bfloat162_rn(v.x - __low2float(hr), v.z - __high2float(hr));
      const __nv_bfloat162 li = __floats2bfloat162_rn(v.y - __low2float(hi), v.w - __high2float(hi));
      *reinterpret_cast<__nv_bfloat162 *>(&Xhi[a * C::SN + gg]) = hr;
      *reinterpret_cast<__nv_bfloat162 *>(&Xhi[(C::D + a) * C::SN + gg]) = hi;
      *reinterpret_cast<__nv_bfloat162 *>(&Xlo[a * C::SN + gg]) = lr;
      *reinterpret_cast<__nv_bfloat162 *>(&Xlo[(C::D + a) * C::SN + gg]) = li;
    }
    __syncthreads();
    float acc[C::NF][4];
#pragma unroll
    for (int nf = 0; nf < C::NF; ++nf) acc[nf][0] = acc[nf][1] = acc[nf][2] = acc[nf][3] = 0.f;
    const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8;  // k row within the k16 step
    const int lcol = (lane >> 4) * 8;                     // n offset: second fragment of the pair
#pragma unroll
    for (int ks = 0; ks < C::KS; ++ks) {
#pragma unroll
      for (int nf = 0; nf < C::NF; nf += 2) {
        const int off = (ks * 16 + lrow) * C::SN + (wn * C::NF + nf) * 8 + lcol;
        uint32_t bh[4], bl[4];
        ldsm_x4_trans(bh, &Xhi[off]);
        ldsm_x4_trans(bl, &Xlo[off]);
        mma_bf16(acc[nf], al[ks], bh[0], bh[1]);
        mma_bf16(acc[nf], ah[ks], bl[0], bl[1]);
        mma_bf16(acc[nf], ah[ks], bh[0], bh[1]);
        mma_bf16(acc[nf + 1], al[ks], bh[2], bh[3]);
        mma_bf16(acc[nf + 1], ah[ks], bl[2], bl[3]);
        mma_bf16(acc[nf + 1], ah[ks], bh[2], bh[3]);
      }
    }
    __syncthreads();  // X is free: the result tile is staged in its place
    // m-tile mt holds Re (rows 0-7) and Im (rows 8-15) of members 8mt..8mt+7
#pragma unroll
    for (int nf = 0; nf < C::NF; ++nf) {
      const int r0 = mt * 16 + (lane >> 2), c0 = (wn * C::NF + nf) * 8 + 2 * (lane & 3);
      *reinterpret_cast<float2 *>(&Ys[r0 * C::SG + c0]) = make_float2(acc[nf][0], acc[nf][1]);
      *reinterpret_cast<float2 *>(&Ys[(r0 + 8) * C::SG + c0]) = make_float2(acc[nf][2], acc[nf][3]);
    }
    __syncthreads();
    const uint64_t g0 = tile * kTcG;
#pragma unroll
    for (int j = 0; j < C::PER; ++j) {
      const int i = threadIdx.x + j * kTcThreads;
      const int gg = i % kTcG, a = i / kTcG;
      const int row = (a >> 3) * 16 + (a & 7);
      const uint64_t g = g0 + gg;
      if (g < n_groups)
        psi[tc_base<K>(g, t) + tc_off<K>(a, t)] =
            make_float2(Ys[row * C::SG + gg], Ys[(row + 8) * C::SG + gg]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
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

template <int K>
bool launch_tc_k(const GateData &g, void *sv, uint32_t n, cudaStream_t s, std::string &err) {
  using C = TcCfg<K>;
  static std::once_flag once;
  static cudaError_t attr_rc = cudaSuccess;
  static int blocks_per_sm = 1;
  std::call_once(once, [] {
    attr_rc = cudaFuncSetAttribute(k_gate_tc<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)C::SMEM);
    if (attr_rc == cudaSuccess)
      attr_rc = cudaFuncSetAttribute(k_gate_tc<K>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_gate_tc<K>, kTcThreads, C::SMEM) ==
            cudaSuccess &&
        b > 0)
      blocks_per_sm = b;
  });
  if (!cuda_ok(attr_rc, "cudaFuncSetAttribute(tensor gate kernel)", err)) return false;
  TcTargets t;
  for (uint32_t b = 0; b < kMaxGateQubits; ++b) {
    const uint32_t q = b < g.k ? g.qubits[b] : 0;
    t.lo_mask[b] = (1ull << q) - 1;
    t.stride[b] = 1ull << q;
  }
  const uint64_t n_groups = 1ull << (n - K);
  const uint64_t n_tiles = (n_groups + kTcG - 1) / kTcG;
  const unsigned grid =
      (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(n_tiles, (uint64_t)blocks_per_sm * sm_count()));
  k_gate_tc<K><<<grid, kTcThreads, C::SMEM, s>>>(static_cast<float2 *>(sv), n_groups, t,
                                                  static_cast<const uint32_t *>(g.d_tc));
  return cuda_ok(cudaGetLastError(), "tensor gate kernel launch", err);
}

}  // namespace

bool tensor_path_supported(const GateData &g) {
  return g.precision == 0 && g.k >= 4 && g.k <= 6;
}

// Packs [[A, -B], [B, A]] (rows permuted as below) into mma.sync m16n8k16 A
// fragments (row-major 16x16 per fragment; a0..a3 = rows gid / gid+8, columns
// 2t..2t+1 / 2t+8..2t+9), hi fragments first, then lo, and uploads them.
bool prepare_tensor_gate(GateData &g, std::string &err) {
  if (!tensor_path_supported(g)) {
    err = "the tensor-core path takes complex64 gates with 4..6 qubits";
    return false;
  }
  const int D = 1 << g.k, R = 2 * D, MT = R / 16, KS = R / 16;
  // Rows are ordered per m16 tile: tile mt = Re rows of members 8mt..8mt+7, then
  // their Im rows; columns are [Re x ; Im x].
  std::vector<double> Mr((size_t)R * R);
  for (int mt = 0; mt < MT; ++mt)
    for (int j = 0; j < 16; ++j) {
      const int r = mt * 8 + (j & 7);  // member
      const bool im = j >= 8;
      double *row = &Mr[(size_t)(mt * 16 + j) * R];
      for (int c = 0; c < D; ++c) {
        const double a = g.m64[2 * (r * D + c)], b = g.m64[2 * (r * D + c) + 1];
        row[c] = im ? b : a;       // x_re coefficient
        row[D + c] = im ? a : -b;  // x_im coefficient
      }
    }
  std::vector<uint16_t> hi((size_t)R * R), lo((size_t)R * R);
  for (size_t i = 0; i < Mr.size(); ++i) {
    hi[i] = bf16_bits_rn((float)Mr[i]);
    lo[i] = bf16_bits_rn((float)(Mr[i] - (double)bf16_value(hi[i])));
  }
  const size_t per = (size_t)MT * KS * 128;  // uint32 per operand
  std::vector<uint32_t> frag(2 * per);
  auto at = [&](const std::vector<uint16_t> &m, int r, int c) -> uint32_t { return m[(size_t)r * R + c]; };
  for (int mt = 0; mt < MT; ++mt)
    for (int ks = 0; ks < KS; ++ks)
      for (int lane = 0; lane < 32; ++lane) {
        const int gid = lane >> 2, tq = lane & 3;
        const int r0 = mt * 16 + gid, c0 = ks * 16 + 2 * tq;
        for (int which = 0; which < 2; ++which) {
          const std::vector<uint16_t> &m = which ? lo : hi;
          uint32_t *dst = frag.data() + which * per + (((size_t)mt * KS + ks) * 32 + lane) * 4;
          dst[0] = at(m, r0, c0) | (at(m, r0, c0 + 1) << 16);
          dst[1] = at(m, r0 + 8, c0) | (at(m, r0 + 8, c0 + 1) << 16);
          dst[2] = at(m, r0, c0 + 8) | (at(m, r0, c0 + 9) << 16);
          dst[3] = at(m, r0 + 8, c0 + 8) | (at(m, r0 + 8, c0 + 9) << 16);
        }
      }
  if (g.d_tc) cudaFree(g.d_tc);
  g.d_tc = nullptr;
  if (!cuda_ok(cudaMalloc(&g.d_tc, frag.size() * 4), "cudaMalloc (tensor gate fragments)", err))
    return false;
  return cuda_ok(cudaMemcpy(g.d_tc, frag.data(), frag.size() * 4, cudaMemcpyHostToDevice),
                 "cudaMemcpy (tensor gate fragments)", err);
}

bool launch_gate_tensor(const GateData &g, void *sv, uint32_t n, cudaStream_t s, std::string &err) {
  if (!g.d_tc || !tensor_path_supported(g)) {
    err = "gate has no tensor-core fragments";
    return false;
  }
  switch (g.k) {
  case 4: return launch_tc_k<4>(g, sv, n, s, err);
  case 5: return launch_tc_k<5>(g, sv, n, s, err);
  default: return launch_tc_k<6>(g, sv, n, s, err);
  }
}

}  // namespace cb2
