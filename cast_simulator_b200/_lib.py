"""ctypes binding of the native library ``libcast_b200.so``.

The library is built in-tree by ``python -m cast_simulator_b200.build``.  There
is no fallback: if the library is missing or fails to load, importing the
package's GPU entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcast_b200.so")
ERR_LEN = 1024

_lib = None

c_u8p = C.POINTER(C.c_uint8)
c_u32p = C.POINTER(C.c_uint32)
c_u64p = C.POINTER(C.c_uint64)
c_dp = C.POINTER(C.c_double)
c_fp = C.POINTER(C.c_float)
c_charpp = C.POINTER(C.c_char_p)


class CudaError(RuntimeError):
    """A failed call through the C ABI (message from the library's err_buf)."""


class Complex64(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class KernelGenSpec(C.Structure):
    """cast_cuda_kernel_gen_spec_t (include/ffi_cuda.h)."""

    _fields_ = [
        ("precision", C.c_int),
        ("ztol", C.c_double),
        ("otol", C.c_double),
        ("sm_major", C.c_uint32),
        ("sm_minor", C.c_uint32),
        ("maxnreg", C.c_uint32),
    ]


class FusionConfigC(C.Structure):
    """cast_b200_fusion_config_t (include/cast_b200.h)."""

    _fields_ = [
        ("size_max", C.c_uint32),
        ("cost_kind", C.c_uint32),
        ("benefit_margin", C.c_double),
        ("zero_tol", C.c_double),
        ("crossover_ai", C.c_double),
        ("tensor_crossover_ai", C.c_double),
        ("tensor_min_k", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


# (name, restype, argtypes) of every exported symbol, in header order.
FFI_CUDA = [
    ("cast_cuda_compile_gate_ptx", C.c_int,
     [C.POINTER(KernelGenSpec), C.POINTER(Complex64), C.c_size_t, c_u32p, C.c_size_t,
      C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), c_u32p, c_u8p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_str_free", None, [C.c_void_p]),
    ("cast_cuda_device_sm", C.c_int, [c_u32p, c_u32p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_free_memory", C.c_int, [c_u64p, c_u64p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_stream_create", C.c_void_p, [C.c_char_p, C.c_size_t]),
    ("cast_cuda_stream_destroy", None, [C.c_void_p]),
    ("cast_cuda_stream_sync", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_ptx_to_cubin", C.c_int,
     [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t]),
    ("cast_cuda_cubin_free", None, [C.c_void_p]),
    ("cast_cuda_cubin_load", C.c_void_p, [C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t]),
    ("cast_cuda_module_unload", None, [C.c_void_p]),
    ("cast_cuda_module_get_function", C.c_void_p,
     [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_kernel_launch", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_cuda_event_create", C.c_void_p, [C.c_char_p, C.c_size_t]),
    ("cast_cuda_event_record", C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_event_synchronize", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_event_destroy", None, [C.c_void_p]),
    ("cast_cuda_event_elapsed_ms", C.c_int,
     [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.c_char_p, C.c_size_t]),
    ("cast_cuda_memcpy_dtod_async", C.c_int,
     [C.c_uint64, C.c_uint64, C.c_size_t, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_cuda_sv_alloc", C.c_uint64, [C.c_size_t, C.c_uint8, C.c_char_p, C.c_size_t]),
    ("cast_cuda_sv_free", None, [C.c_uint64]),
    ("cast_cuda_sv_zero", C.c_int, [C.c_uint64, C.c_size_t, C.c_uint8, C.c_char_p, C.c_size_t]),
    ("cast_cuda_sv_upload", C.c_int,
     [C.c_uint64, c_dp, C.c_size_t, C.c_uint8, C.c_char_p, C.c_size_t]),
    ("cast_cuda_sv_download", C.c_int,
     [C.c_uint64, c_dp, C.c_size_t, C.c_uint8, C.c_char_p, C.c_size_t]),
    ("cast_cuda_norm_squared", C.c_int,
     [C.c_uint64, C.c_size_t, C.c_uint8, c_dp, C.c_char_p, C.c_size_t]),
    ("cast_cuda_scale", C.c_int,
     [C.c_uint64, C.c_size_t, C.c_uint8, C.c_double, C.c_char_p, C.c_size_t]),
]

# Extension entry points (include/cast_b200.h).
CAST_B200 = [
    ("cast_b200_set_device", C.c_int, [C.c_int, C.c_char_p, C.c_size_t]),
    ("cast_b200_stream_create_nonblocking", C.c_void_p, [C.c_char_p, C.c_size_t]),
    ("cast_b200_stream_create_priority", C.c_void_p, [C.c_int, C.c_char_p, C.c_size_t]),
    ("cast_b200_sv_zero_async", C.c_int,
     [C.c_uint64, C.c_size_t, C.c_uint8, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_set_gate_path", C.c_int, [C.c_int]),
    ("cast_b200_set_kernel_choice", C.c_int,
     [C.c_uint8, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_apply_gate", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, C.POINTER(Complex64), c_u32p, C.c_uint32, C.c_double,
      C.c_double, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_program_create", C.c_void_p,
     [C.c_uint8, C.c_uint32, C.c_double, C.c_double, C.c_char_p, C.c_size_t]),
    ("cast_b200_program_add_gate", C.c_int,
     [C.c_void_p, C.POINTER(Complex64), c_u32p, C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_program_set_split_precision", C.c_int,
     [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]),
    ("cast_b200_tensor_status", C.c_int, [C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t]),
    ("cast_b200_set_tensor_loader", C.c_int, [C.c_int]),
    ("cast_b200_program_num_gates", C.c_uint32, [C.c_void_p]),
    ("cast_b200_program_run", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_void_p, C.c_int, C.c_char_p, C.c_size_t]),
    ("cast_b200_program_destroy", None, [C.c_void_p]),
    ("cast_b200_inner_product", C.c_int,
     [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint8, c_dp, c_dp, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_qubit_populations", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, c_dp, c_dp, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_marginal_probabilities", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, c_u32p, C.c_uint32, c_dp, C.c_void_p, C.c_char_p,
      C.c_size_t]),
    ("cast_b200_dm_populations", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, c_dp, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_sample", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, C.c_uint64, C.c_uint64, c_u32p, C.c_uint32, c_u64p,
      C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_sample_at", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, c_dp, C.c_uint64, c_u32p, C.c_uint32, c_u64p, C.c_void_p,
      C.c_char_p, C.c_size_t]),
    ("cast_b200_damping_sums", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, C.c_uint64, C.c_double, c_dp, c_dp, C.c_void_p, C.c_char_p,
      C.c_size_t]),
    ("cast_b200_scale_popc", C.c_int,
     [C.c_uint64, C.c_uint32, C.c_uint8, C.c_uint64, C.c_double, C.c_double, C.c_void_p, C.c_char_p,
      C.c_size_t]),
    ("cast_b200_fuse", C.c_void_p,
     [C.c_uint32, C.c_uint32, c_u32p, c_u32p, C.POINTER(Complex64), C.POINTER(FusionConfigC),
      C.c_char_p, C.c_size_t]),
    ("cast_b200_fused_num_gates", C.c_uint32, [C.c_void_p]),
    ("cast_b200_fused_gate", C.c_int, [C.c_void_p, C.c_uint32, c_u32p, c_u32p, C.POINTER(Complex64)]),
    ("cast_b200_program_add_fused", C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_fused_free", None, [C.c_void_p]),
    ("cast_b200_traj_create", C.c_void_p, [C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_destroy", None, [C.c_void_p]),
    ("cast_b200_traj_add_gate", C.c_int,
     [C.c_void_p, C.POINTER(Complex64), c_u32p, C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_add_pauli_error", C.c_int,
     [C.c_void_p, C.c_double, C.POINTER(Complex64), C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_add_damping", C.c_int,
     [C.c_void_p, C.c_uint32, C.c_double, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_add_channel", C.c_int,
     [C.c_void_p, C.c_uint32, C.POINTER(Complex64), C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_num_ops", C.c_uint32, [C.c_void_p]),
    ("cast_b200_traj_num_qubits", C.c_uint32, [C.c_void_p]),
    ("cast_b200_traj_build", C.c_int,
     [C.c_void_p, C.c_uint32, c_u32p, c_u32p, c_u32p, C.POINTER(Complex64), c_u32p, c_dp, C.c_uint32,
      c_u32p, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_get_op", C.c_int,
     [C.c_void_p, C.c_uint32, c_u32p, c_u32p, c_u32p, c_dp, c_u32p, c_u32p, C.POINTER(Complex64),
      C.c_size_t]),
    ("cast_b200_gate_engine", C.c_int,
     [C.c_uint8, C.c_uint32, C.POINTER(Complex64), c_u32p, C.c_uint32, C.c_double, C.c_double,
      C.c_int, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_set_launch", C.c_int,
     [C.c_void_p, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t]),
    ("cast_b200_traj_run", C.c_int,
     [C.c_void_p, C.c_uint32, C.c_uint64, c_dp, c_u32p, C.c_void_p, C.c_int, C.c_char_p,
      C.c_size_t]),
    ("cast_b200_traj_run_range", C.c_int,
     [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, c_dp, c_u32p, C.c_void_p, C.c_int,
      C.c_char_p, C.c_size_t]),
    ("cast_b200_batch_create", C.c_void_p, [C.c_char_p, C.c_size_t]),
    ("cast_b200_batch_destroy", None, [C.c_void_p]),
    ("cast_b200_batch_add", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint8, C.c_uint32, c_u32p, c_u32p,
      C.POINTER(Complex64), C.c_int, C.c_double, C.c_double, C.c_char_p, C.c_size_t]),
    ("cast_b200_batch_add_fused", C.c_int,
     [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint8, C.c_void_p, C.c_int, C.c_double, C.c_double,
      C.c_char_p, C.c_size_t]),
    ("cast_b200_batch_num_circuits", C.c_uint32, [C.c_void_p]),
    ("cast_b200_batch_num_z", C.c_uint32, [C.c_void_p]),
    ("cast_b200_batch_clear", None, [C.c_void_p]),
    ("cast_b200_batch_run", C.c_int, [C.c_void_p, c_dp, C.c_void_p, C.c_char_p, C.c_size_t]),
    ("cast_b200_norm_squared_noalloc", C.c_int,
     [C.c_uint64, C.c_size_t, C.c_uint8, c_dp, C.c_void_p, C.c_char_p, C.c_size_t]),
]


def lib():
    """Load the native library (raises if it is missing - no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cast_simulator_b200.build`"
            )
        L = C.CDLL(LIB_PATH)
        for name, res, args in FFI_CUDA + CAST_B200:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def errbuf():
    return C.create_string_buffer(ERR_LEN)


def check(rc, eb, what: str = ""):
    if rc != 0:
        msg = eb.value.decode(errors="replace")
        raise CudaError(f"{what}: {msg}" if what else msg)


def check_ptr(p, eb, what: str = ""):
    if not p:
        msg = eb.value.decode(errors="replace")
        raise CudaError(f"{what}: {msg}" if what else msg)
    return p
