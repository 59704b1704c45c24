/*
 * Shared C types of the drop-in C ABI.
 *
 * Layout-identical to the reference header src/cpp/include/ffi_types.h:14-21
 * of narix10yc/cast_simulator (precision enum values and the 16-byte
 * {double re, im} complex), so the reference's Rust FFI declarations
 * (src/ffi/cuda.rs:29-185) bind to this library unchanged.
 */
#ifndef CAST_B200_FFI_TYPES_H
#define CAST_B200_FFI_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces ffi_types.h:14-17 (same values: F32 = 0, F64 = 1). */
typedef enum cast_precision_t {
  CAST_PRECISION_F32 = 0,
  CAST_PRECISION_F64 = 1,
} cast_precision_t;

/* Replaces ffi_types.h:18-21: one complex matrix entry, FP64. */
typedef struct cast_complex64_t {
  double re;
  double im;
} cast_complex64_t;

#ifdef __cplusplus
}
#endif

#endif /* CAST_B200_FFI_TYPES_H */
