// Internal (non-exported) declarations shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace cb2 {

constexpr uint32_t kMaxGateQubits = 7;   // largest fused gate the kernels handle
constexpr uint32_t kMaxSvQubits = 40;    // index math is 64-bit; HBM bounds the rest

// A gate ready for the device: canonical (ascending) qubits and the
// sparsity-snapped matrix in FP64 and FP32 (row-major, interleaved re/im).
struct GateData {
  uint32_t k = 0;
  uint8_t precision = 1;  // 0 = F32, 1 = F64
  uint32_t qubits[kMaxGateQubits] = {0};
  std::vector<double> m64;
  std::vector<float> m32;
  void *d_mat = nullptr;  // device copy in the gate's precision (owned by the holder)
  void *d_tc = nullptr;   // split-BF16 tensor-core gate operand (owned by the holder), if any
  uint32_t tc_k = 0;      // qubits of the tensor-core operand (a 5-qubit gate is padded to 6)
  uint32_t tc_qubits[kMaxGateQubits] = {0};
  void *d_sparse = nullptr;  // CSR copy for the sparse kernel (owned by the holder), if any
};

// Error helper: fills `err` and returns false on a CUDA failure.
inline bool cuda_ok(cudaError_t rc, const char *what, std::string &err) {
  if (rc == cudaSuccess) return true;
  err = std::string(what) + " failed: " + cudaGetErrorName(rc) + " - " + cudaGetErrorString(rc);
  return false;
}

inline void write_err(char *buf, size_t len, const std::string &msg) {
  if (!buf || len == 0) return;
  const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
  std::memcpy(buf, msg.data(), n);
  buf[n] = '\0';
}

inline void clear_err(char *buf, size_t len) {
  if (buf && len) buf[0] = '\0';
}

// Every kernel reads amplitudes as 16-byte vectors (double2 / float4), so a
// device pointer handed in through the C ABI must be 16-byte aligned (every
// cudaMalloc result is 256-byte aligned; an interior pointer may not be).
// Returns false and fills `err` for a misaligned pointer; null passes (the
// callers check for null with their own messages).
inline bool aligned16(uint64_t dptr, const char *what, std::string &err) {
  if ((dptr & 15u) == 0) return true;
  err = std::string(what) + " must be 16-byte aligned (got an address ending in 0x" +
        "0123456789abcdef"[dptr & 15u] + ")";
  return false;
}

// Validates the gate against an n-qubit statevector.
bool check_gate(const GateData &g, uint32_t n, std::string &err);

// Enqueues one gate application on `stream` (in place on `sv`).
bool launch_gate(const GateData &g, void *sv, uint32_t n, cudaStream_t stream, std::string &err);

// Sparse gates (k >= 5, at most 2^k / 4 nonzero entries a row on average after
// snapping) run on the CSR kernel instead of the dense ones; upload_sparse
// fills g.d_sparse.  free_gate_device releases every device copy of a gate.
bool sparse_gate(const GateData &g);

// The kernel family a gate runs on (the same decisions launch_gate takes):
// `tensor` = the gate carries a tensor-core operand, `sparse` = a CSR table.
enum : int {
  kEngineRegister = 0, kEngineTile = 1, kEngineStaged = 2, kEngineSparse = 3,
  kEngineSparseTile = 4, kEngineTensor = 5
};
int gate_engine(const GateData &g, uint32_t n, bool tensor, bool sparse);
bool upload_sparse(GateData &g, std::string &err);
void free_gate_device(GateData &g);

// Classifies matrix scalars as 0 / +-1 / immediate with tolerances scaled by
// 1/2^k and fills g.m64 / g.m32 (src/cpp/cuda/cuda_gen.cpp:84-103).
void snap_matrix(GateData &g, const double *interleaved, double ztol, double otol);

// Tensor-core path (gate_tensor.cu): complex64 gates with 5 or 6 qubits in split
// BF16.  prepare_tensor_gate uploads g.d_tc; launch_gate runs the tensor kernel
// for gates that have it.
bool tensor_path_supported(const GateData &g);
// n: qubits of the statevectors the gate will run on (a spare qubit for padding).
bool prepare_tensor_gate(GateData &g, uint32_t n, std::string &err);
bool launch_gate_tensor(const GateData &g, void *sv, uint32_t n, cudaStream_t s, std::string &err);
// Reads and clears the tensor kernel's error word (nonzero: a bounded wait expired).
bool tensor_error_status(uint32_t *out, std::string &err);
// Tensor-kernel loader: 0 auto (TMA bulk copies where the lowest target is >= 7),
// 1 register loads always, 2 same as auto; returns the previous mode.
int set_tensor_loader(int mode);

// Device helpers shared between translation units.
int sm_count();
int set_gate_path(int path);  // 0 auto, 1 register, 2 tile; returns previous
// Autotuned choice for dense gates of k <= 4 with targets below qubit 5 (see
// cast_b200_set_kernel_choice).
bool set_kernel_choice(uint8_t precision, uint32_t k, uint32_t low_mask, int engine,
                       uint32_t tile_bits, std::string &err);
bool upload_gate_matrix(GateData &g, std::string &err);  // fills g.d_mat

// Reductions (reduce_kernels.cu): synchronous on `s`, except scale (enqueued).
bool norm_squared(const void *x, uint64_t n_scalars, uint8_t precision, double *out,
                  cudaStream_t s, std::string &err);
bool scale(void *x, uint64_t n_scalars, uint8_t precision, double factor, cudaStream_t s,
           std::string &err);
bool inner_product(const void *a, const void *b, uint32_t n, uint8_t precision, double *re,
                   double *im, cudaStream_t s, std::string &err);
bool qubit_populations(const void *x, uint32_t n, uint8_t precision, double *p1, double *norm,
                       cudaStream_t s, std::string &err);
bool marginal_probabilities(const void *x, uint32_t n, uint8_t precision, const uint32_t *measured,
                            uint32_t m, double *out, cudaStream_t s, std::string &err);
bool dm_populations(const void *rho, uint32_t n, uint8_t precision, double *out, cudaStream_t s,
                    std::string &err);
// Amplitude damping on a qubit mask, for host-driven quantum-jump trajectories:
// tot = sum |a_i|^2, wsum = sum |a_i|^2 (1 - gamma)^popc(i & mask) (FP64,
// synchronous); scale_popc multiplies a_i by scale * sfac^popc(i & mask)
// (enqueued on `s`).
bool damping_sums(const void *x, uint32_t n, uint8_t precision, uint64_t mask, double gamma,
                  double *tot, double *wsum, cudaStream_t s, std::string &err);
bool scale_popc(void *x, uint32_t n, uint8_t precision, uint64_t mask, double sfac, double scale,
                cudaStream_t s, std::string &err);

}  // namespace cb2
