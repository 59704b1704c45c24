// The drop-in C ABI of include/ffi_cuda.h.
//
// Replaces the reference's CUDA executor and gate compiler
// (src/cpp/cuda/ffi_cuda.cpp:69-147, src/cpp/cuda/cuda_exec.cpp:104-533 of
// narix10yc/cast_simulator) with the same entry points, argument meaning,
// ownership rules and error convention, but no runtime code generation:
//
//   compile_gate_ptx  -> validated, sparsity-snapped gate descriptor (text)
//   ptx_to_cubin      -> the descriptor's binary form
//   cubin_load        -> a Module owning the device copy of the matrix
//   module_get_function -> the Module's dispatch handle
//   kernel_launch     -> precompiled sm_100a kernel for (precision, k)
//
// All calls use the CUDA runtime on the calling thread's current device (the
// primary context, shared with PyTorch and any other runtime user).
#include "../../include/ffi_cuda.h"
#include "internal.hpp"

#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <exception>
#include <new>
#include <sstream>

using cb2::clear_err;
using cb2::cuda_ok;
using cb2::GateData;
using cb2::write_err;

namespace {

constexpr char kEntryName[] = "k_gate";
constexpr char kBlobMagic[8] = {'C', 'B', '2', 'G', 'A', 'T', 'E', '1'};
constexpr uint32_t kModuleMagic = 0xCB200A11u;
constexpr uint32_t kFunctionMagic = 0xCB200F11u;

struct BlobHeader {
  char magic[8];
  uint32_t version;
  uint32_t k;
  uint32_t precision;
  uint32_t qubits[cb2::kMaxGateQubits];
  uint64_t n_scalars;
  char entry[16];
};

struct Module;
struct Function {
  uint32_t magic = kFunctionMagic;
  Module *module = nullptr;
};

struct Module {
  uint32_t magic = kModuleMagic;
  GateData gate;
  Function fn;
};

// Make sure a device is usable; the first runtime call creates the context.
bool ensure_cuda(std::string &err) {
  int n = 0;
  cudaError_t rc = cudaGetDeviceCount(&n);
  if (!cuda_ok(rc, "cudaGetDeviceCount", err)) return false;
  if (n == 0) {
    err = "no CUDA device is visible";
    return false;
  }
  return cuda_ok(cudaFree(nullptr), "CUDA context initialisation", err);
}

char *dup_cstr(const std::string &s) {
  char *p = new char[s.size() + 1];
  std::memcpy(p, s.data(), s.size());
  p[s.size()] = '\0';
  return p;
}

std::string descriptor_text(const GateData &g) {
  std::ostringstream os;
  os << "// cast_b200 gate descriptor: consumed by cast_cuda_ptx_to_cubin, not PTX\n";
  os << ".cast_b200 1\n";
  os << ".entry " << kEntryName << "\n";
  os << ".precision " << (g.precision ? "f64" : "f32") << "\n";
  os << ".k " << g.k << "\n.qubits";
  for (uint32_t b = 0; b < g.k; ++b) os << ' ' << g.qubits[b];
  os << "\n.matrix";
  char buf[24];
  for (double v : g.m64) {
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    std::snprintf(buf, sizeof(buf), " %016" PRIx64, bits);
    os << buf;
  }
  os << "\n";
  return os.str();
}

bool parse_descriptor(const char *text, GateData &g, std::string &err) {
  std::istringstream is(text);
  std::string line;
  bool have_magic = false, have_k = false, have_q = false, have_m = false, have_p = false;
  while (std::getline(is, line)) {
    if (line.empty() || line[0] == '/') continue;
    std::istringstream ls(line);
    std::string key;
    ls >> key;
    if (key == ".cast_b200") {
      int v = 0;
      ls >> v;
      have_magic = (v == 1);
    } else if (key == ".entry") {
      std::string e;
      ls >> e;
      if (e != kEntryName) {
        err = "descriptor names unknown entry '" + e + "'";
        return false;
      }
    } else if (key == ".precision") {
      std::string p;
      ls >> p;
      if (p == "f64") g.precision = 1;
      else if (p == "f32") g.precision = 0;
      else {
        err = "descriptor has invalid precision '" + p + "'";
        return false;
      }
      have_p = true;
    } else if (key == ".k") {
      ls >> g.k;
      have_k = true;
    } else if (key == ".qubits") {
      if (!have_k || g.k == 0 || g.k > cb2::kMaxGateQubits) {
        err = "descriptor has an invalid gate size";
        return false;
      }
      for (uint32_t b = 0; b < g.k; ++b)
        if (!(ls >> g.qubits[b])) {
          err = "descriptor qubit list is truncated";
          return false;
        }
      have_q = true;
    } else if (key == ".matrix") {
      if (!have_k) {
        err = "descriptor matrix precedes its size";
        return false;
      }
      const size_t ns = 2ull << (2 * g.k);
      g.m64.resize(ns);
      g.m32.resize(ns);
      std::string tok;
      for (size_t i = 0; i < ns; ++i) {
        if (!(ls >> tok) || tok.size() != 16) {
          err = "descriptor matrix is truncated";
          return false;
        }
        const uint64_t bits = std::strtoull(tok.c_str(), nullptr, 16);
        double v;
        std::memcpy(&v, &bits, 8);
        g.m64[i] = v;
        g.m32[i] = (float)v;
      }
      have_m = true;
    }
  }
  if (!have_magic || !have_k || !have_q || !have_m || !have_p) {
    err = "not a cast_b200 gate descriptor";
    return false;
  }
  return true;
}

size_t scalar_bytes(uint8_t precision) { return precision == 0 ? sizeof(float) : sizeof(double); }

}  // namespace

// Shared with the extension TU (cast_b200_*): module -> gate.
namespace cb2 {
bool upload_gate_matrix(GateData &g, std::string &err) {
  const size_t ns = g.m64.size();
  const size_t bytes = ns * (g.precision ? sizeof(double) : sizeof(float));
  if (!cuda_ok(cudaMalloc(&g.d_mat, bytes), "cudaMalloc (gate matrix)", err)) return false;
  const void *src = g.precision ? (const void *)g.m64.data() : (const void *)g.m32.data();
  if (!cuda_ok(cudaMemcpy(g.d_mat, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy (gate matrix)",
               err)) {
    cudaFree(g.d_mat);
    g.d_mat = nullptr;
    return false;
  }
  return true;
}


const GateData *module_gate(const void *fn_or_module) {
  if (!fn_or_module) return nullptr;
  const uint32_t magic = *static_cast<const uint32_t *>(fn_or_module);
  if (magic == kFunctionMagic) return &static_cast<const Function *>(fn_or_module)->module->gate;
  if (magic == kModuleMagic) return &static_cast<const Module *>(fn_or_module)->gate;
  return nullptr;
}
}  // namespace cb2

extern "C" {

// ── gate "compilation" (replaces ffi_cuda.cpp:69-145) ─────────────────────────

int cast_cuda_compile_gate_ptx(const cast_cuda_kernel_gen_spec_t *spec,
                               const cast_complex64_t *matrix, size_t matrix_len,
                               const uint32_t *qubits, size_t n_qubits, char **out_ptx,
                               char **out_func_name, uint32_t *out_n_gate_qubits,
                               uint8_t *out_precision, char *err_buf, size_t err_buf_len) {
  if (!spec || !matrix || !qubits || !out_ptx || !out_func_name || !out_n_gate_qubits ||
      !out_precision) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  try {
    if (spec->precision != CAST_PRECISION_F32 && spec->precision != CAST_PRECISION_F64) {
      write_err(err_buf, err_buf_len, "spec.precision must be F32 or F64");
      return 1;
    }
    if (n_qubits == 0) {
      write_err(err_buf, err_buf_len, "qubits must not be null/empty");
      return 1;
    }
    if (n_qubits > cb2::kMaxGateQubits) {
      write_err(err_buf, err_buf_len,
                "gates on more than " + std::to_string(cb2::kMaxGateQubits) +
                    " qubits are not supported (fuse with size_max <= 7)");
      return 1;
    }
    if (matrix_len != (1ull << (2 * n_qubits))) {
      write_err(err_buf, err_buf_len, "matrixLen must equal (2^nQubits)^2");
      return 1;
    }
    GateData g;
    g.k = (uint32_t)n_qubits;
    g.precision = spec->precision == CAST_PRECISION_F64 ? 1 : 0;
    for (size_t b = 0; b < n_qubits; ++b) {
      g.qubits[b] = qubits[b];
      if (b && qubits[b - 1] >= qubits[b]) {
        write_err(err_buf, err_buf_len, "qubits must be distinct and ascending");
        return 1;
      }
    }
    cb2::snap_matrix(g, reinterpret_cast<const double *>(matrix), spec->ztol, spec->otol);
    *out_ptx = dup_cstr(descriptor_text(g));
    *out_func_name = dup_cstr(kEntryName);
    *out_n_gate_qubits = g.k;
    *out_precision = g.precision;
    clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  } catch (...) {
    write_err(err_buf, err_buf_len, "unknown error in gate compilation");
    return 1;
  }
}

void cast_cuda_str_free(const char *s) { delete[] s; }

// ── device queries (cuda_exec.cpp:106-153) ───────────────────────────────────

int cast_cuda_device_sm(uint32_t *out_major, uint32_t *out_minor, char *err_buf,
                        size_t err_buf_len) {
  std::string err;
  if (!ensure_cuda(err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  int dev = 0, major = 0, minor = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice", err) ||
      !cuda_ok(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev),
               "cudaDeviceGetAttribute (major)", err) ||
      !cuda_ok(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev),
               "cudaDeviceGetAttribute (minor)", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  if (out_major) *out_major = (uint32_t)major;
  if (out_minor) *out_minor = (uint32_t)minor;
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_cuda_free_memory(uint64_t *out_free_bytes, uint64_t *out_total_bytes, char *err_buf,
                          size_t err_buf_len) {
  std::string err;
  size_t f = 0, t = 0;
  if (!ensure_cuda(err) || !cuda_ok(cudaMemGetInfo(&f, &t), "cudaMemGetInfo", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  if (out_free_bytes) *out_free_bytes = f;
  if (out_total_bytes) *out_total_bytes = t;
  clear_err(err_buf, err_buf_len);
  return 0;
}

// ── streams (cuda_exec.cpp:268-298) ──────────────────────────────────────────

void *cast_cuda_stream_create(char *err_buf, size_t err_buf_len) {
  std::string err;
  cudaStream_t s = nullptr;
  if (!ensure_cuda(err) ||
      !cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamDefault), "cudaStreamCreate", err)) {
    write_err(err_buf, err_buf_len, err);
    return nullptr;
  }
  clear_err(err_buf, err_buf_len);
  return s;
}

void cast_cuda_stream_destroy(void *stream) {
  if (stream) cudaStreamDestroy(static_cast<cudaStream_t>(stream));
}

int cast_cuda_stream_sync(void *stream, char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!cuda_ok(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "cudaStreamSynchronize",
               err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

// ── descriptor -> blob (replaces cuda_exec.cpp:157-219) ──────────────────────

int cast_cuda_ptx_to_cubin(const char *ptx_data, uint8_t **out_cubin, size_t *out_cubin_len,
                           char *err_buf, size_t err_buf_len) {
  if (!ptx_data || !out_cubin || !out_cubin_len) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  try {
    GateData g;
    std::string err;
    if (!parse_descriptor(ptx_data, g, err)) {
      write_err(err_buf, err_buf_len, err);
      return 1;
    }
    BlobHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kBlobMagic, 8);
    h.version = 1;
    h.k = g.k;
    h.precision = g.precision;
    for (uint32_t b = 0; b < g.k; ++b) h.qubits[b] = g.qubits[b];
    h.n_scalars = g.m64.size();
    std::memcpy(h.entry, kEntryName, sizeof(kEntryName));
    const size_t len = sizeof(h) + g.m64.size() * sizeof(double);
    uint8_t *buf = new uint8_t[len];
    std::memcpy(buf, &h, sizeof(h));
    std::memcpy(buf + sizeof(h), g.m64.data(), g.m64.size() * sizeof(double));
    *out_cubin = buf;
    *out_cubin_len = len;
    clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
}

void cast_cuda_cubin_free(const uint8_t *cubin) { delete[] cubin; }

// ── modules (replaces cuda_exec.cpp:223-264) ─────────────────────────────────

void *cast_cuda_cubin_load(const uint8_t *cubin_data, size_t cubin_len, char *err_buf,
                           size_t err_buf_len) {
  if (!cubin_data) {
    write_err(err_buf, err_buf_len, "cubinData must not be null");
    return nullptr;
  }
  // The caller passes the blob's full length (the reference's Rust caller hands
  // over cubin.len(), cuda/kernel.rs:313-319); nothing is read beyond it, so a
  // length of 0 or one shorter than the header is refused before any read.
  if (cubin_len < sizeof(BlobHeader)) {
    write_err(err_buf, err_buf_len, "gate module is truncated (shorter than its header)");
    return nullptr;
  }
  try {
    BlobHeader h;
    std::memcpy(&h, cubin_data, sizeof(h));
    if (std::memcmp(h.magic, kBlobMagic, 8) != 0 || h.version != 1 || h.k == 0 ||
        h.k > cb2::kMaxGateQubits || h.precision > 1 || h.n_scalars != (2ull << (2 * h.k))) {
      write_err(err_buf, err_buf_len, "not a cast_b200 gate module");
      return nullptr;
    }
    if (cubin_len < sizeof(h) + h.n_scalars * sizeof(double)) {
      write_err(err_buf, err_buf_len, "gate module is truncated");
      return nullptr;
    }
    std::string err;
    if (!ensure_cuda(err)) {
      write_err(err_buf, err_buf_len, err);
      return nullptr;
    }
    Module *m = new Module;
    m->fn.module = m;
    m->gate.k = h.k;
    m->gate.precision = (uint8_t)h.precision;
    for (uint32_t b = 0; b < h.k; ++b) m->gate.qubits[b] = h.qubits[b];
    m->gate.m64.resize(h.n_scalars);
    std::memcpy(m->gate.m64.data(), cubin_data + sizeof(h), h.n_scalars * sizeof(double));
    m->gate.m32.resize(h.n_scalars);
    for (size_t i = 0; i < h.n_scalars; ++i) m->gate.m32[i] = (float)m->gate.m64[i];
    if (!cb2::upload_gate_matrix(m->gate, err) ||
        (cb2::sparse_gate(m->gate) && !cb2::upload_sparse(m->gate, err))) {
      cb2::free_gate_device(m->gate);
      delete m;
      write_err(err_buf, err_buf_len, err);
      return nullptr;
    }
    clear_err(err_buf, err_buf_len);
    return m;
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return nullptr;
  }
}

void cast_cuda_module_unload(void *cu_module) {
  Module *m = static_cast<Module *>(cu_module);
  if (!m || m->magic != kModuleMagic) return;
  cb2::free_gate_device(m->gate);
  m->magic = 0;
  delete m;
}

void *cast_cuda_module_get_function(void *cu_module, const char *func_name, char *err_buf,
                                    size_t err_buf_len) {
  Module *m = static_cast<Module *>(cu_module);
  if (!m || !func_name) {
    write_err(err_buf, err_buf_len, "cuModule and funcName must not be null");
    return nullptr;
  }
  if (m->magic != kModuleMagic) {
    write_err(err_buf, err_buf_len, "invalid module handle");
    return nullptr;
  }
  if (std::strcmp(func_name, kEntryName) != 0) {
    write_err(err_buf, err_buf_len, std::string("named symbol not found: ") + func_name);
    return nullptr;
  }
  clear_err(err_buf, err_buf_len);
  return &m->fn;
}

// ── launch (replaces cuda_exec.cpp:302-335) ──────────────────────────────────

int cast_cuda_kernel_launch(void *cu_function, void *stream, uint64_t sv_dptr,
                            uint32_t n_gate_qubits, uint32_t sv_n_qubits, char *err_buf,
                            size_t err_buf_len) {
  if (!cu_function) {
    write_err(err_buf, err_buf_len, "cuFunction must not be null");
    return 1;
  }
  Function *f = static_cast<Function *>(cu_function);
  if (f->magic != kFunctionMagic || !f->module) {
    write_err(err_buf, err_buf_len, "invalid function handle");
    return 1;
  }
  if (sv_n_qubits < n_gate_qubits) {
    write_err(err_buf, err_buf_len, "statevector has fewer qubits than the gate kernel requires");
    return 1;
  }
  const GateData &g = f->module->gate;
  if (n_gate_qubits != g.k) {
    write_err(err_buf, err_buf_len, "n_gate_qubits does not match the gate module");
    return 1;
  }
  std::string err;
  if (!cb2::launch_gate(g, reinterpret_cast<void *>(sv_dptr), sv_n_qubits,
                        static_cast<cudaStream_t>(stream), err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

// ── events (cuda_exec.cpp:339-405) ───────────────────────────────────────────

void *cast_cuda_event_create(char *err_buf, size_t err_buf_len) {
  std::string err;
  cudaEvent_t ev = nullptr;
  if (!ensure_cuda(err) || !cuda_ok(cudaEventCreate(&ev), "cudaEventCreate", err)) {
    write_err(err_buf, err_buf_len, err);
    return nullptr;
  }
  clear_err(err_buf, err_buf_len);
  return ev;
}

int cast_cuda_event_record(void *event, void *stream, char *err_buf, size_t err_buf_len) {
  if (!event || !stream) {
    write_err(err_buf, err_buf_len, "event and stream must not be null");
    return 1;
  }
  std::string err;
  if (!cuda_ok(cudaEventRecord(static_cast<cudaEvent_t>(event), static_cast<cudaStream_t>(stream)),
               "cudaEventRecord", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_cuda_event_synchronize(void *event, char *err_buf, size_t err_buf_len) {
  if (!event) {
    write_err(err_buf, err_buf_len, "event must not be null");
    return 1;
  }
  std::string err;
  if (!cuda_ok(cudaEventSynchronize(static_cast<cudaEvent_t>(event)), "cudaEventSynchronize",
               err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

void cast_cuda_event_destroy(void *event) {
  if (event) cudaEventDestroy(static_cast<cudaEvent_t>(event));
}

int cast_cuda_event_elapsed_ms(void *start_event, void *end_event, float *out_ms, char *err_buf,
                               size_t err_buf_len) {
  if (!start_event || !end_event || !out_ms) {
    write_err(err_buf, err_buf_len, "arguments must not be null");
    return 1;
  }
  std::string err;
  if (!cuda_ok(cudaEventElapsedTime(out_ms, static_cast<cudaEvent_t>(start_event),
                                    static_cast<cudaEvent_t>(end_event)),
               "cudaEventElapsedTime", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

// ── device-to-device copy (cuda_exec.cpp:409-425) ────────────────────────────

int cast_cuda_memcpy_dtod_async(uint64_t dst, uint64_t src, size_t n_bytes, void *stream,
                                char *err_buf, size_t err_buf_len) {
  std::string err;
  if (!ensure_cuda(err) ||
      !cuda_ok(cudaMemcpyAsync(reinterpret_cast<void *>(dst), reinterpret_cast<const void *>(src),
                               n_bytes, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)),
               "cudaMemcpyAsync (DtoD)", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

// ── statevector memory (cuda_exec.cpp:429-533) ───────────────────────────────

uint64_t cast_cuda_sv_alloc(size_t n_elements, uint8_t precision, char *err_buf,
                            size_t err_buf_len) {
  std::string err;
  void *p = nullptr;
  if (!ensure_cuda(err) ||
      !cuda_ok(cudaMalloc(&p, n_elements * scalar_bytes(precision)), "cudaMalloc", err)) {
    write_err(err_buf, err_buf_len, err);
    return 0;
  }
  clear_err(err_buf, err_buf_len);
  return reinterpret_cast<uint64_t>(p);
}

void cast_cuda_sv_free(uint64_t dptr) {
  if (dptr) cudaFree(reinterpret_cast<void *>(dptr));
}

int cast_cuda_sv_zero(uint64_t dptr, size_t n_elements, uint8_t precision, char *err_buf,
                      size_t err_buf_len) {
  std::string err;
  void *d = reinterpret_cast<void *>(dptr);
  const size_t sb = scalar_bytes(precision);
  if (!cuda_ok(cudaMemset(d, 0, n_elements * sb), "cudaMemset", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  const float one32 = 1.0f;
  const double one64 = 1.0;
  if (n_elements > 0 &&
      !cuda_ok(cudaMemcpy(d, precision == 0 ? (const void *)&one32 : (const void *)&one64, sb,
                          cudaMemcpyHostToDevice),
               "cudaMemcpy (zero state)", err)) {
    write_err(err_buf, err_buf_len, err);
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_cuda_sv_upload(uint64_t dptr, const double *host_data, size_t n_elements,
                        uint8_t precision, char *err_buf, size_t err_buf_len) {
  std::string err;
  if (n_elements && (!dptr || !host_data)) {
    write_err(err_buf, err_buf_len, "sv upload: null device or host pointer");
    return 1;
  }
  try {
    if (precision != 0) {
      if (!cuda_ok(cudaMemcpy(reinterpret_cast<void *>(dptr), host_data, n_elements * 8,
                              cudaMemcpyHostToDevice),
                   "cudaMemcpy (upload)", err)) {
        write_err(err_buf, err_buf_len, err);
        return 1;
      }
    } else {
      const size_t chunk = 1u << 24;
      std::vector<float> tmp(std::min(chunk, n_elements));
      for (size_t off = 0; off < n_elements; off += chunk) {
        const size_t cnt = std::min(chunk, n_elements - off);
        for (size_t i = 0; i < cnt; ++i) tmp[i] = (float)host_data[off + i];
        if (!cuda_ok(cudaMemcpy(reinterpret_cast<float *>(dptr) + off, tmp.data(), cnt * 4,
                                cudaMemcpyHostToDevice),
                     "cudaMemcpy (upload f32)", err)) {
          write_err(err_buf, err_buf_len, err);
          return 1;
        }
      }
    }
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

int cast_cuda_sv_download(uint64_t dptr, double *host_data, size_t n_elements, uint8_t precision,
                          char *err_buf, size_t err_buf_len) {
  std::string err;
  if (n_elements && (!dptr || !host_data)) {
    write_err(err_buf, err_buf_len, "sv download: null device or host pointer");
    return 1;
  }
  try {
    if (precision != 0) {
      if (!cuda_ok(cudaMemcpy(host_data, reinterpret_cast<const void *>(dptr), n_elements * 8,
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy (download)", err)) {
        write_err(err_buf, err_buf_len, err);
        return 1;
      }
    } else {
      const size_t chunk = 1u << 24;
      std::vector<float> tmp(std::min(chunk, n_elements));
      for (size_t off = 0; off < n_elements; off += chunk) {
        const size_t cnt = std::min(chunk, n_elements - off);
        if (!cuda_ok(cudaMemcpy(tmp.data(), reinterpret_cast<const float *>(dptr) + off, cnt * 4,
                                cudaMemcpyDeviceToHost),
                     "cudaMemcpy (download f32)", err)) {
          write_err(err_buf, err_buf_len, err);
          return 1;
        }
        for (size_t i = 0; i < cnt; ++i) host_data[off + i] = (double)tmp[i];
      }
    }
  } catch (const std::exception &ex) {
    write_err(err_buf, err_buf_len, ex.what());
    return 1;
  }
  clear_err(err_buf, err_buf_len);
  return 0;
}

}  // extern "C"
