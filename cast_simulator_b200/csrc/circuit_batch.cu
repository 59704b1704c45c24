// Many small circuits in one persistent launch.
//
// The reference simulates one circuit at a time: Simulator::simulate launches
// one kernel per gate on the whole device and synchronises
// (src/simulator/mod.rs:523-547; cuda_exec.cpp:302-335).  For circuits of up to
// ~16 qubits a gate pass is a few microseconds of work spread over 148 SMs, so
// such a stream is bound by launches and host round trips.  Here a batch of
// independent circuits - different qubit counts, depths and precisions - runs
// in ONE launch:
//
//  * a persistent grid of CTAs (512 threads); each CTA claims the next circuit
//    from a device work counter, so long and short circuits balance (the host
//    orders the batch longest first);
//  * the CTA owns the circuit's statevector (the caller's device buffer, at
//    most 2^20 amplitudes: 16 MiB in complex128) and runs every fused gate
//    (k <= 4) on it in place, one thread per gather group, a __syncthreads()
//    between gates; the gate matrix is staged in shared memory first.  Small
//    states stay in L1/L2 across the whole circuit;
//  * optionally it starts from |0...0> (written by the CTA itself);
//  * at the end it reduces, in FP64 and in a fixed order, the norm and
//    P(q = 1) of every qubit, and writes <Z_q> = (norm - 2 P(q = 1)) / norm.
//
// Matrices are snapped with the plain path's zero / +-1 rule
// (src/cpp/cuda/cuda_gen.cpp:84-103) and stored in the circuit's precision.
// Everything a batch needs - circuit table, op list, matrices, the work
// counter - is packed into one pinned host buffer and sent with one copy; the
// <Z> table comes back with one copy: three operations on one stream a batch.
#include "../../include/cast_b200.h"
#include "internal.hpp"

#include <algorithm>
#include <cstring>
#include <exception>
#include <mutex>
#include <numeric>
#include <vector>

namespace {

using cb2::cuda_ok;
using cb2::write_err;
using cb2::clear_err;

constexpr int kBThreads = 512;
constexpr uint32_t kBatchMaxQubits = 20;
constexpr uint32_t kBatchMaxGate = 4;
constexpr uint32_t kBatchMagic = 0xB47C4001u;

struct BCircuit {
  uint64_t sv;      // device statevector (interleaved re/im)
  uint32_t n;       // qubits
  uint32_t prec;    // 0 = F32, 1 = F64
  uint32_t op_begin;
  uint32_t n_ops;
  uint32_t init_zero;
  uint32_t z_off;   // first <Z> slot of this circuit
};

struct BOp {
  uint32_t k;
  uint32_t q[kBatchMaxGate];
  uint32_t mat;  // byte offset of the matrix in the pool (16-byte aligned)
};

struct BHeader {
  uint32_t next;  // work counter (zero in every upload)
  uint32_t n_circuits;
  uint32_t n_ops;
  uint32_t pad;
};

template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };

template <typename V> __device__ __forceinline__ V cmac(V m, V x, V acc) {
  acc.x = fma(m.x, x.x, acc.x);
  acc.x = fma(-m.y, x.y, acc.x);
  acc.y = fma(m.x, x.y, acc.y);
  acc.y = fma(m.y, x.x, acc.y);
  return acc;
}

// One fused k-qubit gate applied in place: thread t takes groups t, t + 512, ...
template <typename T, int K>
__device__ __noinline__ void batch_gate(typename C2<T>::type *sv, uint32_t n, const uint32_t *q,
                                        const typename C2<T>::type *M) {
  using V = typename C2<T>::type;
  constexpr int D = 1 << K;
  uint32_t lo[K];
#pragma unroll
  for (int b = 0; b < K; ++b) lo[b] = (1u << q[b]) - 1;
  const uint32_t ng = 1u << (n - K);
  for (uint32_t g = threadIdx.x; g < ng; g += kBThreads) {
    uint32_t base = g;
#pragma unroll
    for (int b = 0; b < K; ++b) base = ((base & ~lo[b]) << 1) | (base & lo[b]);
    V x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      uint32_t o = base;
#pragma unroll
      for (int b = 0; b < K; ++b)
        if ((a >> b) & 1) o += lo[b] + 1;
      x[a] = sv[o];
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
      V acc;
      acc.x = 0;
      acc.y = 0;
#pragma unroll
      for (int c = 0; c < D; ++c) acc = cmac(M[r * D + c], x[c], acc);
      uint32_t o = base;
#pragma unroll
      for (int b = 0; b < K; ++b)
        if ((r >> b) & 1) o += lo[b] + 1;
      sv[o] = acc;
    }
  }
}

struct BShared {
  double2 mat[1u << (2 * kBatchMaxGate)];  // 4 KiB: the largest matrix in complex128
  double red[kBThreads / 32][kBatchMaxQubits + 1];
  BCircuit circ;
  uint32_t claim;
};

template <typename T>
__device__ void run_circuit(BShared &S, const BOp *__restrict__ ops, const char *__restrict__ pool,
                            double *__restrict__ out_z) {
  using V = typename C2<T>::type;
  const BCircuit c = S.circ;
  V *sv = reinterpret_cast<V *>(c.sv);
  const uint32_t N = 1u << c.n;
  if (c.init_zero) {
    for (uint32_t i = threadIdx.x; i < N; i += kBThreads) {
      V v;
      v.x = i == 0 ? (T)1 : (T)0;
      v.y = 0;
      sv[i] = v;
    }
    __syncthreads();
  }
  V *Msm = reinterpret_cast<V *>(S.mat);
  for (uint32_t oi = 0; oi < c.n_ops; ++oi) {
    const BOp op = ops[c.op_begin + oi];
    const V *Mg = reinterpret_cast<const V *>(pool + op.mat);
    const uint32_t entries = 1u << (2 * op.k);
    for (uint32_t i = threadIdx.x; i < entries; i += kBThreads) Msm[i] = Mg[i];
    __syncthreads();
    switch (op.k) {
    case 1: batch_gate<T, 1>(sv, c.n, op.q, Msm); break;
    case 2: batch_gate<T, 2>(sv, c.n, op.q, Msm); break;
    case 3: batch_gate<T, 3>(sv, c.n, op.q, Msm); break;
    default: batch_gate<T, 4>(sv, c.n, op.q, Msm); break;
    }
    __syncthreads();
  }
  // FP64 norm and P(q = 1) per qubit, reduced in a fixed order
  double acc[kBatchMaxQubits + 1];
#pragma unroll
  for (uint32_t q = 0; q <= kBatchMaxQubits; ++q) acc[q] = 0.0;
  for (uint32_t i = threadIdx.x; i < N; i += kBThreads) {
    const V v = sv[i];
    const double p = (double)v.x * v.x + (double)v.y * v.y;
    acc[kBatchMaxQubits] += p;
#pragma unroll
    for (uint32_t q = 0; q < kBatchMaxQubits; ++q)
      if ((i >> q) & 1) acc[q] += p;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (uint32_t q = 0; q <= kBatchMaxQubits; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) S.red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < c.n) {
    double tot = 0.0, p1 = 0.0;
    for (int w = 0; w < kBThreads / 32; ++w) {
      tot += S.red[w][kBatchMaxQubits];
      p1 += S.red[w][threadIdx.x];
    }
    out_z[c.z_off + threadIdx.x] = tot > 0.0 ? (tot - 2.0 * p1) / tot : 0.0;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kBThreads, 1)
    k_circuit_batch(BHeader *__restrict__ hdr, const BCircuit *__restrict__ circs,
                    const BOp *__restrict__ ops, const char *__restrict__ pool,
                    double *__restrict__ out_z) {
  __shared__ BShared S;
  const uint32_t n_circ = hdr->n_circuits;
  while (true) {
    if (threadIdx.x == 0) {
      S.claim = atomicAdd(&hdr->next, 1u);
      if (S.claim < n_circ) S.circ = circs[S.claim];
    }
    __syncthreads();
    if (S.claim >= n_circ) return;
    if (S.circ.prec == 1) run_circuit<double>(S, ops, pool, out_z);
    else run_circuit<float>(S, ops, pool, out_z);
  }
}

// ── host side ────────────────────────────────────────────────────────────────

struct Batch {
  uint32_t magic = kBatchMagic;
  std::mutex mu;
  std::vector<BCircuit> circs;
  std::vector<BOp> ops;
  std::vector<char> pool;   // matrices, each 16-byte aligned
  std::vector<uint64_t> cost;  // work estimate per circuit (ordering)
  uint32_t n_z = 0;
  // device and pinned buffers, grown on demand and reused across runs
  char *dev = nullptr;
  size_t dev_cap = 0;
  char *host = nullptr;
  size_t host_cap = 0;
  double *host_z = nullptr;
  size_t host_z_cap = 0;
  int device = -1;

  ~Batch() {
    if (dev) cudaFree(dev);
    if (host) cudaFreeHost(host);
    if (host_z) cudaFreeHost(host_z);
  }
};

Batch *as_batch(void *p) {
  Batch *b = static_cast<Batch *>(p);
  return b && b->magic == kBatchMagic ? b : nullptr;
}

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

bool add_circuit(Batch &b, uint64_t sv, uint32_t n, uint8_t prec, uint32_t n_gates,
                 const uint32_t *gate_k, const uint32_t *qubits, const double *mats, int init_zero,
                 double ztol, double otol, std::string &err) {
  if (!sv) {
    err = "statevector must not be null";
    return false;
  }
  if (!cb2::aligned16(sv, "statevector pointer", err)) return false;
  if (prec > 1 || n == 0 || n > kBatchMaxQubits) {
    err = "batched circuits: precision 0 / 1 and 1.." + std::to_string(kBatchMaxQubits) + " qubits";
    return false;
  }
  if (n_gates && (!gate_k || !qubits || !mats)) {
    err = "gate arrays must not be null";
    return false;
  }
  BCircuit c{};
  c.sv = sv;
  c.n = n;
  c.prec = prec;
  c.op_begin = (uint32_t)b.ops.size();
  c.n_ops = n_gates;
  c.init_zero = init_zero ? 1 : 0;
  c.z_off = b.n_z;
  std::vector<BOp> new_ops;
  std::vector<char> new_pool;
  size_t qoff = 0, moff = 0;
  uint64_t cost = 0;
  for (uint32_t i = 0; i < n_gates; ++i) {
    const uint32_t k = gate_k[i];
    if (k == 0 || k > kBatchMaxGate || k > n) {
      err = "batched circuits take gates of 1.." + std::to_string(kBatchMaxGate) +
            " qubits within the circuit (gate " + std::to_string(i) + ")";
      return false;
    }
    cb2::GateData g;
    g.k = k;
    g.precision = prec;
    BOp op{};
    op.k = k;
    for (uint32_t j = 0; j < k; ++j) {
      const uint32_t q = qubits[qoff + j];
      if (q >= n || (j && qubits[qoff + j - 1] >= q)) {
        err = "gate " + std::to_string(i) + ": qubits must be ascending and below the circuit's size";
        return false;
      }
      op.q[j] = q;
    }
    qoff += k;
    const size_t entries = 1ull << (2 * k);
    cb2::snap_matrix(g, mats + 2 * moff, ztol, otol);
    moff += entries;
    const size_t bytes = entries * (prec ? 16 : 8);
    op.mat = (uint32_t)(b.pool.size() + new_pool.size());
    const size_t at = new_pool.size();
    new_pool.resize(align16(at + bytes));
    if (prec) std::memcpy(new_pool.data() + at, g.m64.data(), bytes);
    else std::memcpy(new_pool.data() + at, g.m32.data(), bytes);
    new_ops.push_back(op);
    cost += (uint64_t)entries << (n - k);  // complex multiply-adds of the pass
  }
  if (b.pool.size() + new_pool.size() > 0xFFFFFFF0ull) {
    err = "batch matrix pool exceeds 4 GiB";
    return false;
  }
  b.ops.insert(b.ops.end(), new_ops.begin(), new_ops.end());
  b.pool.insert(b.pool.end(), new_pool.begin(), new_pool.end());
  b.circs.push_back(c);
  b.cost.push_back(cost + (2ull << n));
  b.n_z += n;
  return true;
}

bool run_batch(Batch &b, double *out_z, cudaStream_t s, std::string &err) {
  const uint32_t nc = (uint32_t)b.circs.size();
  if (nc == 0) return true;
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", err)) return false;
  if (b.device != dev) {  // buffers belong to the device they were made on
    if (b.dev) cudaFree(b.dev);
    b.dev = nullptr;
    b.dev_cap = 0;
    b.device = dev;
  }
  // longest first: the work counter hands them out in this order
  std::vector<uint32_t> order(nc);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t c) { return b.cost[a] > b.cost[c]; });
  const size_t off_c = align16(sizeof(BHeader));
  const size_t off_o = align16(off_c + sizeof(BCircuit) * nc);
  const size_t off_p = align16(off_o + sizeof(BOp) * b.ops.size());
  const size_t off_z = align16(off_p + b.pool.size());
  const size_t up = off_z, total = off_z + sizeof(double) * b.n_z;
  if (b.dev_cap < total) {
    if (b.dev) cudaFree(b.dev);
    b.dev = nullptr;
    const size_t cap = std::max(total, b.dev_cap * 2);
    if (!cuda_ok(cudaMalloc(&b.dev, cap), "cudaMalloc (circuit batch)", err)) {
      b.dev_cap = 0;
      return false;
    }
    b.dev_cap = cap;
  }
  if (b.host_cap < up) {
    if (b.host) cudaFreeHost(b.host);
    b.host = nullptr;
    const size_t cap = std::max(up, b.host_cap * 2);
    if (!cuda_ok(cudaMallocHost(&b.host, cap), "cudaMallocHost (circuit batch)", err)) {
      b.host_cap = 0;
      return false;
    }
    b.host_cap = cap;
  }
  if (b.host_z_cap < b.n_z) {
    if (b.host_z) cudaFreeHost(b.host_z);
    b.host_z = nullptr;
    const size_t cap = std::max<size_t>(b.n_z, b.host_z_cap * 2);
    if (!cuda_ok(cudaMallocHost(&b.host_z, cap * sizeof(double)), "cudaMallocHost (batch <Z>)", err)) {
      b.host_z_cap = 0;
      return false;
    }
    b.host_z_cap = cap;
  }
  BHeader h{0u, nc, (uint32_t)b.ops.size(), 0u};
  std::memcpy(b.host, &h, sizeof(h));
  BCircuit *hc = reinterpret_cast<BCircuit *>(b.host + off_c);
  for (uint32_t i = 0; i < nc; ++i) hc[i] = b.circs[order[i]];
  std::memcpy(b.host + off_o, b.ops.data(), sizeof(BOp) * b.ops.size());
  std::memcpy(b.host + off_p, b.pool.data(), b.pool.size());
  int per_sm = 1;
  if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_circuit_batch, kBThreads, 0),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor", err))
    return false;
  const uint32_t slots = (uint32_t)std::max(1, per_sm) * (uint32_t)std::max(1, cb2::sm_count());
  const unsigned grid = (unsigned)std::min<uint32_t>(nc, slots);
  bool ok = cuda_ok(cudaMemcpyAsync(b.dev, b.host, up, cudaMemcpyHostToDevice, s),
                    "cudaMemcpyAsync (batch upload)", err);
  if (ok) {
    k_circuit_batch<<<grid, kBThreads, 0, s>>>(
        reinterpret_cast<BHeader *>(b.dev), reinterpret_cast<const BCircuit *>(b.dev + off_c),
        reinterpret_cast<const BOp *>(b.dev + off_o), b.dev + off_p,
        reinterpret_cast<double *>(b.dev + off_z));
    ok = cuda_ok(cudaGetLastError(), "circuit batch launch", err) &&
         cuda_ok(cudaMemcpyAsync(b.host_z, b.dev + off_z, sizeof(double) * b.n_z,
                                 cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync (batch <Z>)", err);
  }
  // the pinned buffers are reused by the next run: wait for the copies either way
  std::string e2;
  const bool synced = cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize (circuit batch)", e2);
  if (ok && !synced) err = e2;
  ok = ok && synced;
  if (ok && out_z) std::memcpy(out_z, b.host_z, sizeof(double) * b.n_z);
  return ok;
}

bool check_distinct(const Batch &b, std::string &err) {
  std::vector<std::pair<uint64_t, uint64_t>> spans;  // [begin, end) bytes of each statevector
  for (const BCircuit &c : b.circs)
    spans.emplace_back(c.sv, c.sv + ((uint64_t)(c.prec ? 16 : 8) << c.n));
  std::sort(spans.begin(), spans.end());
  for (size_t i = 1; i < spans.size(); ++i)
    if (spans[i].first < spans[i - 1].second) {
      err = "two circuits of a batch share statevector memory";
      return false;
    }
  return true;
}

}  // namespace

extern "C" {

void *cast_b200_batch_create(char *err_buf, size_t err_buf_len) {
  try {
    Batch *b = new Batch;
    clear_err(err_buf, err_buf_len);
    return b;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return nullptr;
  }
}

void cast_b200_batch_destroy(void *batch) {
  Batch *b = as_batch(batch);
  if (!b) return;
  b->magic = 0;
  delete b;
}

int cast_b200_batch_add(void *batch, uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                        uint32_t n_gates, const uint32_t *gate_k, const uint32_t *qubits,
                        const cast_complex64_t *matrices, int init_zero, double ztol, double otol,
                        char *err_buf, size_t err_buf_len) {
  Batch *b = as_batch(batch);
  if (!b) {
    write_err(err_buf, err_buf_len, "invalid batch handle");
    return 1;
  }
  try {
    std::lock_guard<std::mutex> lock(b->mu);
    std::string err;
    if (!add_circuit(*b, sv_dptr, n_qubits, precision, n_gates, gate_k, qubits,
                     reinterpret_cast<const double *>(matrices), init_zero, ztol, otol, err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_batch_add_fused(void *batch, uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                              const void *fused, int init_zero, double ztol, double otol,
                              char *err_buf, size_t err_buf_len) {
  Batch *b = as_batch(batch);
  if (!b || !fused) {
    write_err(err_buf, err_buf_len, "invalid batch or fused-circuit handle");
    return 1;
  }
  try {
    const uint32_t ng = cast_b200_fused_num_gates(fused);
    std::vector<uint32_t> ks(ng), qs;
    std::vector<cast_complex64_t> ms;
    for (uint32_t i = 0; i < ng; ++i) {
      uint32_t k = 0, q[cb2::kMaxGateQubits] = {0};
      if (cast_b200_fused_gate(fused, i, &k, q, nullptr) || k == 0 || k > kBatchMaxGate) {
        write_err(err_buf, err_buf_len,
                  "fused gate " + std::to_string(i) + " is wider than the batch kernel's " +
                      std::to_string(kBatchMaxGate) + " qubits (fuse with size_max <= 4)");
        return 1;
      }
      const size_t at = ms.size();
      ms.resize(at + (1ull << (2 * k)));
      cast_b200_fused_gate(fused, i, &k, q, ms.data() + at);
      ks[i] = k;
      qs.insert(qs.end(), q, q + k);
    }
    std::lock_guard<std::mutex> lock(b->mu);
    std::string err;
    if (!add_circuit(*b, sv_dptr, n_qubits, precision, ng, ks.data(), qs.data(),
                     reinterpret_cast<const double *>(ms.data()), init_zero, ztol, otol, err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

uint32_t cast_b200_batch_num_circuits(const void *batch) {
  const Batch *b = static_cast<const Batch *>(batch);
  return b && b->magic == kBatchMagic ? (uint32_t)b->circs.size() : 0;
}

uint32_t cast_b200_batch_num_z(const void *batch) {
  const Batch *b = static_cast<const Batch *>(batch);
  return b && b->magic == kBatchMagic ? b->n_z : 0;
}

void cast_b200_batch_clear(void *batch) {
  Batch *b = as_batch(batch);
  if (!b) return;
  std::lock_guard<std::mutex> lock(b->mu);
  b->circs.clear();
  b->ops.clear();
  b->pool.clear();
  b->cost.clear();
  b->n_z = 0;
}

int cast_b200_batch_run(void *batch, double *out_z, void *stream, char *err_buf,
                        size_t err_buf_len) {
  Batch *b = as_batch(batch);
  if (!b) {
    write_err(err_buf, err_buf_len, "invalid batch handle");
    return 1;
  }
  try {
    std::lock_guard<std::mutex> lock(b->mu);
    std::string err;
    if (!check_distinct(*b, err) || !run_batch(*b, out_z, static_cast<cudaStream_t>(stream), err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

}  // extern "C"
