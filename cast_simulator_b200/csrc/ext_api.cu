// Extension C ABI (include/cast_b200.h): one-call gate application, gate
// programs replayed through CUDA graphs, and FP64 reductions.
#include "../../include/cast_b200.h"
#include "internal.hpp"

#include <algorithm>

#include <exception>
#include <map>
#include <mutex>
#include <utility>

using cb2::clear_err;
using cb2::cuda_ok;
using cb2::GateData;
using cb2::write_err;

namespace {

constexpr uint32_t kProgramMagic = 0xCB2009A1u;

bool make_gate(uint8_t precision, const cast_complex64_t *matrix, const uint32_t *qubits,
               uint32_t k, double ztol, double otol, GateData &g, std::string &err) {
  if (!matrix || !qubits) {
    err = "matrix and qubits must not be null";
    return false;
  }
  if (precision > 1) {
    err = "precision must be 0 (F32) or 1 (F64)";
    return false;
  }
  if (k == 0 || k > cb2::kMaxGateQubits) {
    err = "gate must act on 1.." + std::to_string(cb2::kMaxGateQubits) + " qubits";
    return false;
  }
  g.k = k;
  g.precision = precision;
  for (uint32_t b = 0; b < k; ++b) {
    g.qubits[b] = qubits[b];
    if (b && qubits[b - 1] >= qubits[b]) {
      err = "qubits must be distinct and ascending";
      return false;
    }
  }
  cb2::snap_matrix(g, reinterpret_cast<const double *>(matrix), ztol, otol);
  return true;
}

struct Program {
  uint32_t magic = kProgramMagic;
  uint8_t precision = 1;
  uint32_t n = 0;
  double ztol = 0, otol = 0;
  bool split = false;  // complex64 gates with 4..6 qubits run on the tensor cores
  std::vector<GateData> gates;
  std::map<std::pair<uint64_t, void *>, cudaGraphExec_t> graphs;
  std::mutex mu;

  ~Program() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto &g : gates) cb2::free_gate_device(g);
  }

  void drop_graphs() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }

  bool launch_all(uint64_t sv, cudaStream_t s, std::string &err) {
    for (auto &g : gates)
      if (!cb2::launch_gate(g, reinterpret_cast<void *>(sv), n, s, err)) return false;
    return true;
  }
};

Program *as_program(void *p) {
  Program *pr = static_cast<Program *>(p);
  return pr && pr->magic == kProgramMagic ? pr : nullptr;
}

__global__ void k_set_one(void *p, int f64) {
  if (f64) *static_cast<double *>(p) = 1.0;
  else *static_cast<float *>(p) = 1.0f;
}

}  // namespace

extern "C" {

void *cast_b200_stream_create_nonblocking(char *err_buf, size_t err_buf_len) {
  std::string err;
  cudaStream_t s = nullptr;
  if (!cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate", err)) {
    write_err(err_buf, err_buf_len, err);
    return nullptr;
  }
  clear_err(err_buf, err_buf_len);
  return s;
}

void *cast_b200_stream_create_priority(int priority, char *err_buf, size_t err_buf_len) {
  std::string err;
  int least = 0, greatest = 0;
  cudaStream_t s = nullptr;
  if (!cuda_ok(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange",
               err)) {
    write_err(err_buf, err_buf_len, err);
    return nullptr;
  }
  // numerically lower is more urgent; clamp into the device's range
  const int p = std::min(std::max(priority, greatest), least);
  if (!cuda_ok(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, p),
               "cudaStreamCreateWithPriority", err)) {
    write_err(err_buf, err_buf_len, err);
    return nullptr;
  }
  clear_err(err_buf, err_buf_len);
  return s;
}

int cast_b200_sv_zero_async(uint64_t dptr, size_t n_elements, uint8_t precision, void *stream,
                            char *err_buf, size_t err_buf_len) {
  std::string err;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void *d = reinterpret_cast<void *>(dptr);
  if (!d || precision > 1) {
    write_err(err_buf, err_buf_len, "invalid statevector or precision");
    return 1;
  }
  const size_t sb = precision ? sizeof(double) : sizeof(float);
  if (!cuda_ok(cudaMemsetAsync(d, 0, n_elements * sb, s), "cudaMemsetAsync", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  if (n_elements) {
    k_set_one<<<1, 1, 0, s>>>(d, precision);
    if (!cuda_ok(cudaGetLastError(), "zero-state kernel launch", err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_set_device(int device, char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_set_gate_path(int path) { return cb2::set_gate_path(path); }

int cast_b200_set_kernel_choice(uint8_t precision, uint32_t k, uint32_t low_mask, int engine,
                                uint32_t tile_bits, char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!cb2::set_kernel_choice(precision, k, low_mask, engine, tile_bits, err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_gate_engine(uint8_t precision, uint32_t sv_n_qubits, const cast_complex64_t *matrix,
                          const uint32_t *qubits, uint32_t n_gate_qubits, double ztol,
                          double otol, int split, char *err_buf, size_t err_buf_len) {
  try {
    GateData g;
    std::string err;
    if (!make_gate(precision, matrix, qubits, n_gate_qubits, ztol, otol, g, err) ||
        !cb2::check_gate(g, sv_n_qubits, err)) {
      write_err(err_buf, err_buf_len, err);
      return -1;
    }
    const bool sparse = cb2::sparse_gate(g);
    const bool tensor = !sparse && split && cb2::tensor_path_supported(g);
    clear_err(err_buf, err_buf_len);
    return cb2::gate_engine(g, sv_n_qubits, tensor, sparse);
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return -1;
  }
}

int cast_b200_apply_gate(uint64_t sv_dptr, uint32_t sv_n_qubits, uint8_t precision,
                         const cast_complex64_t *matrix, const uint32_t *qubits,
                         uint32_t n_gate_qubits, double ztol, double otol, void *stream,
                         char *err_buf, size_t err_buf_len) {
  try {
    GateData g;
    std::string err;
    if (!make_gate(precision, matrix, qubits, n_gate_qubits, ztol, otol, g, err) ||
        !cb2::check_gate(g, sv_n_qubits, err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool ok;
    const bool sparse = cb2::sparse_gate(g);
    if (sparse || g.k >= 6) {
      // the device copy is freed once the launch that reads it has finished
      ok = (sparse ? cb2::upload_sparse(g, err) : cb2::upload_gate_matrix(g, err)) &&
           cb2::launch_gate(g, reinterpret_cast<void *>(sv_dptr), sv_n_qubits, s, err) &&
           cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize", err);
      cb2::free_gate_device(g);
    } else {
      ok = cb2::launch_gate(g, reinterpret_cast<void *>(sv_dptr), sv_n_qubits, s, err);
    }
    if (!ok) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
    clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
}

void *cast_b200_program_create(uint8_t precision, uint32_t sv_n_qubits, double ztol, double otol,
                               char *err_buf, size_t err_buf_len) {
  if (precision > 1 || sv_n_qubits == 0 || sv_n_qubits > cb2::kMaxSvQubits) {
    write_err(err_buf, err_buf_len, "invalid precision or statevector size");
    return nullptr;
  }
  try {
    Program *p = new Program;
    p->precision = precision;
    p->n = sv_n_qubits;
    p->ztol = ztol;
    p->otol = otol;
    clear_err(err_buf, err_buf_len);
    return p;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return nullptr;
  }
}

int cast_b200_program_add_gate(void *program, const cast_complex64_t *matrix,
                               const uint32_t *qubits, uint32_t n_gate_qubits, char *err_buf,
                               size_t err_buf_len) {
  Program *p = as_program(program);
  if (!p) {
    write_err(err_buf, err_buf_len, "invalid program handle");
    return 1;
  }
  try {
    GateData g;
    std::string err;
    bool ok = make_gate(p->precision, matrix, qubits, n_gate_qubits, p->ztol, p->otol, g, err) &&
              cb2::check_gate(g, p->n, err);
    if (ok) {
      if (cb2::sparse_gate(g)) ok = cb2::upload_sparse(g, err);  // CSR kernel, any precision mode
      else
        ok = (g.k < 6 || cb2::upload_gate_matrix(g, err)) &&
             (!p->split || !cb2::tensor_path_supported(g) || cb2::prepare_tensor_gate(g, p->n, err));
    }
    if (!ok) {
      cb2::free_gate_device(g);
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
    std::lock_guard<std::mutex> lock(p->mu);
    p->drop_graphs();
    p->gates.push_back(std::move(g));
    clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
}

int cast_b200_program_set_split_precision(void *program, int enable, char *err_buf,
                                          size_t err_buf_len) {
  Program *p = as_program(program);
  if (!p) {
    write_err(err_buf, err_buf_len, "invalid program handle");
    return 1;
  }
  std::lock_guard<std::mutex> lock(p->mu);
  if (!p->gates.empty()) {
    write_err(err_buf, err_buf_len, "set the split-precision mode before adding gates");
    return 1;
  }
  p->split = enable != 0;
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_set_tensor_loader(int mode) { return cb2::set_tensor_loader(mode); }

int cast_b200_tensor_status(uint32_t *out_bits, char *err_buf, size_t err_buf_len) {
  if (!out_bits) {
    write_err(err_buf, err_buf_len, "out_bits is null");
    return 1;
  }
  std::string err;
  if (!cb2::tensor_error_status(out_bits, err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

uint32_t cast_b200_program_num_gates(const void *program) {
  const Program *p = static_cast<const Program *>(program);
  return p && p->magic == kProgramMagic ? (uint32_t)p->gates.size() : 0;
}

int cast_b200_program_run(void *program, uint64_t sv_dptr, void *stream, int use_graph,
                          char *err_buf, size_t err_buf_len) {
  Program *p = as_program(program);
  if (!p || !sv_dptr) {
    write_err(err_buf, err_buf_len, "invalid program handle or statevector");
    return 1;
  }
  {
    std::string err;
    if (!cb2::aligned16(sv_dptr, "statevector pointer", err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
  }
  try {
    std::lock_guard<std::mutex> lock(p->mu);
    std::string err;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!use_graph || !s || p->gates.empty()) {
      if (!p->launch_all(sv_dptr, s, err)) {
        write_err(err_buf, err_buf_len, err);
        return 1;
      }
      clear_err(err_buf, err_buf_len);
      return 0;
    }
    auto key = std::make_pair(sv_dptr, stream);
    auto it = p->graphs.find(key);
    if (it == p->graphs.end()) {
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      if (!cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal),
                   "cudaStreamBeginCapture", err)) {
        write_err(err_buf, err_buf_len, err);
        return 1;
      }
      const bool launched = p->launch_all(sv_dptr, s, err);
      const cudaError_t end_rc = cudaStreamEndCapture(s, &graph);
      if (!launched || !cuda_ok(end_rc, "cudaStreamEndCapture", err) ||
          !cuda_ok(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate", err)) {
        if (graph) cudaGraphDestroy(graph);
        write_err(err_buf, err_buf_len, err);
        return 1;
      }
      cudaGraphDestroy(graph);
      it = p->graphs.emplace(key, exec).first;
    }
    if (!cuda_ok(cudaGraphLaunch(it->second, s), "cudaGraphLaunch", err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
    clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
}

void cast_b200_program_destroy(void *program) {
  Program *p = as_program(program);
  if (!p) return;
  p->magic = 0;
  delete p;
}

int cast_b200_inner_product(uint64_t a_dptr, uint64_t b_dptr, uint32_t n_qubits,
                            uint8_t precision, double *out_re, double *out_im, void *stream,
                            char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!out_re || !out_im || !a_dptr || !b_dptr) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  if (!cb2::inner_product(reinterpret_cast<const void *>(a_dptr),
                          reinterpret_cast<const void *>(b_dptr), n_qubits, precision, out_re,
                          out_im, static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_qubit_populations(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                                double *out_p1, double *out_norm, void *stream, char *err_buf,
                                size_t err_buf_len) {
  std::string err;
  if (!out_p1 || !sv_dptr) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  if (!cb2::qubit_populations(reinterpret_cast<const void *>(sv_dptr), n_qubits, precision, out_p1,
                              out_norm, static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_marginal_probabilities(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                                     const uint32_t *measured, uint32_t n_measured,
                                     double *out_probs, void *stream, char *err_buf,
                                     size_t err_buf_len) {
  std::string err;
  if (!out_probs || !measured || !sv_dptr) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  if (!cb2::marginal_probabilities(reinterpret_cast<const void *>(sv_dptr), n_qubits, precision,
                                   measured, n_measured, out_probs,
                                   static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_damping_sums(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t mask,
                           double gamma, double *out_total, double *out_weighted, void *stream,
                           char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!sv_dptr || !out_total || !out_weighted) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  if (!cb2::damping_sums(reinterpret_cast<const void *>(sv_dptr), n_qubits, precision, mask, gamma,
                         out_total, out_weighted, static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_scale_popc(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t mask,
                         double factor, double scale, void *stream, char *err_buf,
                         size_t err_buf_len) {
  std::string err;
  if (!sv_dptr) {
    write_err(err_buf, err_buf_len, "statevector must not be null");
    return 1;
  }
  if (!cb2::scale_popc(reinterpret_cast<void *>(sv_dptr), n_qubits, precision, mask, factor, scale,
                       static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_b200_dm_populations(uint64_t rho_dptr, uint32_t n_physical, uint8_t precision,
                             double *out, void *stream, char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!out || !rho_dptr) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  if (!cb2::dm_populations(reinterpret_cast<const void *>(rho_dptr), n_physical, precision, out,
                           static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

}  // extern "C"
