/*
 * Drop-in C ABI of the CUDA gate-application backend.
 *
 * Every declaration below replaces the one of the same name in the reference
 * header src/cpp/include/ffi_cuda.h of narix10yc/cast_simulator (line numbers
 * cited per entry), with the same argument meaning, ownership and error
 * convention: int 0 = success / 1 = failure (or NULL / 0 for handle- and
 * pointer-returning calls); on failure a NUL-terminated message is written to
 * err_buf (the Rust caller passes 1024 bytes), on success err_buf[0] = '\0'.
 * No C++ exception crosses this boundary.
 *
 * What changes behind the boundary: there is no LLVM/NVPTX JIT.  The
 * "PTX" returned by cast_cuda_compile_gate_ptx is a textual gate descriptor
 * (precision, target qubits, the sparsity-snapped matrix) and the "cubin" is
 * its binary form; cast_cuda_cubin_load uploads the matrix and returns a module
 * whose single function dispatches to precompiled sm_100a kernels specialised
 * on (precision, k).  The Rust side treats both blobs as opaque bytes
 * (src/cuda/kernel.rs:366-488), so it needs no change.
 */
#ifndef CAST_B200_FFI_CUDA_H
#define CAST_B200_FFI_CUDA_H

#include "ffi_types.h"

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces ffi_cuda.h:16-23; layout-compatible with the Rust #[repr(C)]
 * CudaKernelGenSpec (src/cuda/types.rs:10-26).  sm_major/sm_minor/maxnreg are
 * accepted and recorded but do not change code generation (kernels are
 * precompiled for sm_100a). */
typedef struct cast_cuda_kernel_gen_spec_t {
  cast_precision_t precision;
  double ztol;
  double otol;
  uint32_t sm_major;
  uint32_t sm_minor;
  uint32_t maxnreg;
} cast_cuda_kernel_gen_spec_t;

/* -- Gate "compilation" -------------------------------------------------- */

/* Replaces ffi_cuda.h:27-31.  Validates the gate, classifies each matrix
 * scalar as 0 / +1 / -1 / immediate with tolerances ztol/2^k and otol/2^k
 * (the rule of src/cpp/cuda/cuda_gen.cpp:84-103) and returns a descriptor
 * string in *out_ptx and the entry name in *out_func_name (both freed with
 * cast_cuda_str_free).  Reentrant; needs no GPU. */
int cast_cuda_compile_gate_ptx(const cast_cuda_kernel_gen_spec_t *spec,
                               const cast_complex64_t *matrix, size_t matrix_len,
                               const uint32_t *qubits, size_t n_qubits, char **out_ptx,
                               char **out_func_name, uint32_t *out_n_gate_qubits,
                               uint8_t *out_precision, char *err_buf, size_t err_buf_len);
/* Replaces ffi_cuda.h:32. */
void cast_cuda_str_free(const char *s);

/* -- Device capability query -------------------------------------------- */

/* Replaces ffi_cuda.h:36-37 (compute capability of the current device). */
int cast_cuda_device_sm(uint32_t *out_major, uint32_t *out_minor, char *err_buf,
                        size_t err_buf_len);
/* Replaces ffi_cuda.h:38-39. */
int cast_cuda_free_memory(uint64_t *out_free_bytes, uint64_t *out_total_bytes, char *err_buf,
                          size_t err_buf_len);

/* -- Streams ------------------------------------------------------------- */

/* Replaces ffi_cuda.h:43 (a blocking stream, like CU_STREAM_DEFAULT). */
void *cast_cuda_stream_create(char *err_buf, size_t err_buf_len);
/* Replaces ffi_cuda.h:44. */
void cast_cuda_stream_destroy(void *stream);
/* Replaces ffi_cuda.h:45. */
int cast_cuda_stream_sync(void *stream, char *err_buf, size_t err_buf_len);

/* -- Descriptor -> loadable blob ----------------------------------------- */

/* Replaces ffi_cuda.h:49-50: parses the descriptor text into a binary blob
 * (new[]'d, freed with cast_cuda_cubin_free). */
int cast_cuda_ptx_to_cubin(const char *ptx_data, uint8_t **out_cubin, size_t *out_cubin_len,
                           char *err_buf, size_t err_buf_len);
/* Replaces ffi_cuda.h:51. */
void cast_cuda_cubin_free(const uint8_t *cubin);

/* -- Module loading and launch ------------------------------------------- */

/* Replaces ffi_cuda.h:55-56: uploads the gate matrix to the device and
 * returns a module handle owning it. */
void *cast_cuda_cubin_load(const uint8_t *cubin_data, size_t cubin_len, char *err_buf,
                           size_t err_buf_len);
/* Replaces ffi_cuda.h:57. */
void cast_cuda_module_unload(void *cu_module);
/* Replaces ffi_cuda.h:58-59: returns the module's dispatch handle when
 * func_name matches the descriptor's entry name. */
void *cast_cuda_module_get_function(void *cu_module, const char *func_name, char *err_buf,
                                    size_t err_buf_len);
/* Replaces ffi_cuda.h:60-62: applies the gate in place to the 2^sv_n_qubits
 * statevector at sv_dptr (interleaved re/im of the module's precision) on
 * `stream` (NULL = legacy default stream).  Asynchronous. */
int cast_cuda_kernel_launch(void *cu_function, void *stream, uint64_t sv_dptr,
                            uint32_t n_gate_qubits, uint32_t sv_n_qubits, char *err_buf,
                            size_t err_buf_len);

/* -- Timing events -------------------------------------------------------- */

/* Replace ffi_cuda.h:66-71. */
void *cast_cuda_event_create(char *err_buf, size_t err_buf_len);
int cast_cuda_event_record(void *event, void *stream, char *err_buf, size_t err_buf_len);
int cast_cuda_event_synchronize(void *event, char *err_buf, size_t err_buf_len);
void cast_cuda_event_destroy(void *event);
int cast_cuda_event_elapsed_ms(void *start_event, void *end_event, float *out_ms, char *err_buf,
                               size_t err_buf_len);

/* -- Device-to-device copy ------------------------------------------------ */

/* Replaces ffi_cuda.h:75-76. */
int cast_cuda_memcpy_dtod_async(uint64_t dst, uint64_t src, size_t n_bytes, void *stream,
                                char *err_buf, size_t err_buf_len);

/* -- Statevector memory ----------------------------------------------------
 * n_elements counts scalars (2 per amplitude); precision 0 = F32, 1 = F64.
 * Replace ffi_cuda.h:80-89 (cuda_exec.cpp:429-533).  For F32 the host FP64
 * data is narrowed on upload and widened on download, in bounded chunks. */
uint64_t cast_cuda_sv_alloc(size_t n_elements, uint8_t precision, char *err_buf,
                            size_t err_buf_len);
void cast_cuda_sv_free(uint64_t dptr);
int cast_cuda_sv_zero(uint64_t dptr, size_t n_elements, uint8_t precision, char *err_buf,
                      size_t err_buf_len);
int cast_cuda_sv_upload(uint64_t dptr, const double *host_data, size_t n_elements,
                        uint8_t precision, char *err_buf, size_t err_buf_len);
int cast_cuda_sv_download(uint64_t dptr, double *host_data, size_t n_elements, uint8_t precision,
                          char *err_buf, size_t err_buf_len);

/* -- Device reductions ----------------------------------------------------- */

/* Replaces ffi_cuda.h:95-96 (cuda_kernels.cu:244-248): sum of squares of all
 * n_elements scalars, accumulated in FP64; synchronous. */
int cast_cuda_norm_squared(uint64_t dptr, size_t n_elements, uint8_t precision, double *out_norm_sq,
                           char *err_buf, size_t err_buf_len);
/* Replaces ffi_cuda.h:99-100 (cuda_kernels.cu:250-254): x *= scale, enqueued
 * on the legacy default stream. */
int cast_cuda_scale(uint64_t dptr, size_t n_elements, uint8_t precision, double scale,
                    char *err_buf, size_t err_buf_len);

#ifdef __cplusplus
}
#endif

#endif /* CAST_B200_FFI_CUDA_H */
