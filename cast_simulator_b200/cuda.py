"""Host-side mirror of the reference's CUDA backend managers, over the C ABI.

Mirrors src/cuda/{types,statevector,kernel,mod}.rs of narix10yc/cast_simulator:
``CudaKernelGenSpec`` (types.rs:10-56), ``CudaStatevector`` (statevector.rs:52-252),
``CudaKernelManager`` with ``generate`` / ``apply`` / ``sync``
(kernel.rs:778-977), ``device_sm`` and ``cuda_free_memory_bytes``
(mod.rs:38-73).  Every call goes through the drop-in ``ffi_cuda.h`` entry
points of ``libcast_b200.so`` exactly as the Rust code calls the reference's.
"""
from __future__ import annotations

import ctypes as C
import enum
import hashlib
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


class CudaPrecision(enum.IntEnum):
    F32 = 0
    F64 = 1

    def scalar_bytes(self) -> int:
        return 4 if self == CudaPrecision.F32 else 8


def device_sm() -> tuple[int, int]:
    """(major, minor) of the current device (mod.rs:38-60)."""
    eb = L.errbuf()
    ma, mi = C.c_uint32(), C.c_uint32()
    L.check(L.lib().cast_cuda_device_sm(C.byref(ma), C.byref(mi), eb, L.ERR_LEN), eb, "device_sm")
    return ma.value, mi.value


def set_device(device: int) -> None:
    """Make ``device`` current for this host thread (cudaSetDevice)."""
    eb = L.errbuf()
    L.check(L.lib().cast_b200_set_device(int(device), eb, L.ERR_LEN), eb, "set_device")


def cuda_free_memory_bytes() -> tuple[int, int]:
    """(free, total) device memory in bytes (mod.rs:62-73)."""
    eb = L.errbuf()
    f, t = C.c_uint64(), C.c_uint64()
    L.check(L.lib().cast_cuda_free_memory(C.byref(f), C.byref(t), eb, L.ERR_LEN), eb, "free_memory")
    return f.value, t.value


@dataclass
class CudaKernelGenSpec:
    """types.rs:10-56: precision, zero/one tolerances, SM version, maxnreg."""

    precision: CudaPrecision = CudaPrecision.F64
    ztol: float = 1e-12
    otol: float = 1e-12
    sm_major: int = 10
    sm_minor: int = 0
    maxnreg: int = 128

    @classmethod
    def f64(cls) -> "CudaKernelGenSpec":
        return cls(CudaPrecision.F64, 1e-12, 1e-12)

    @classmethod
    def f32(cls) -> "CudaKernelGenSpec":
        return cls(CudaPrecision.F32, 1e-6, 1e-6)

    def to_c(self) -> L.KernelGenSpec:
        return L.KernelGenSpec(int(self.precision), self.ztol, self.otol, self.sm_major,
                               self.sm_minor, self.maxnreg)


class CudaStatevector:
    """Device statevector: interleaved re/im, 2 * 2^n scalars (statevector.rs:52-57)."""

    def __init__(self, n_qubits: int, precision: CudaPrecision = CudaPrecision.F64):
        self._n = int(n_qubits)
        self._prec = CudaPrecision(precision)
        self._len = 2 << self._n
        self._release = None
        eb = L.errbuf()
        self._dptr = L.lib().cast_cuda_sv_alloc(self._len, int(self._prec), eb, L.ERR_LEN)
        if not self._dptr:
            raise L.CudaError(f"allocating {n_qubits}-qubit statevector: {eb.value.decode()}")

    def __del__(self):
        p = getattr(self, "_dptr", 0)
        if p:
            release = getattr(self, "_release", None)
            try:
                if release is not None and release(self._n, self._prec, p, self._len):
                    self._dptr = 0
                    return
                L.lib().cast_cuda_sv_free(p)
            except Exception:
                pass
            self._dptr = 0

    @classmethod
    def _adopt(cls, n_qubits: int, precision: CudaPrecision, dptr: int, release=None) -> "CudaStatevector":
        """Wrap an allocation handed back by a memory pool; ``release(n, prec,
        dptr, len)`` is offered the allocation when this object dies (returns
        True to keep it)."""
        sv = cls.__new__(cls)
        sv._n, sv._prec, sv._len, sv._dptr = int(n_qubits), CudaPrecision(precision), 2 << int(n_qubits), dptr
        sv._release = release
        return sv

    def n_qubits(self) -> int:
        return self._n

    def precision(self) -> CudaPrecision:
        return self._prec

    def __len__(self) -> int:
        return self._len

    @property
    def dptr(self) -> int:
        return self._dptr

    def nbytes(self) -> int:
        return self._len * self._prec.scalar_bytes()

    def zero(self, stream=None) -> None:
        """Reset to |0...0>: host-synchronous (cast_cuda_sv_zero) without a
        stream, ordered on `stream` (a Stream or a raw handle) with one."""
        eb = L.errbuf()
        if stream is None:
            L.check(L.lib().cast_cuda_sv_zero(self._dptr, self._len, int(self._prec), eb, L.ERR_LEN),
                    eb, "sv zero")
            return
        h = getattr(stream, "handle", stream)
        L.check(L.lib().cast_b200_sv_zero_async(self._dptr, self._len, int(self._prec), h, eb,
                                                L.ERR_LEN), eb, "sv zero async")

    def upload(self, amps) -> None:
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128))
        if a.shape != (1 << self._n,):
            raise ValueError(f"expected {1 << self._n} amplitudes, got {a.shape}")
        buf = a.view(np.float64)
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_sv_upload(self._dptr, buf.ctypes.data_as(L.c_dp), self._len,
                                            int(self._prec), eb, L.ERR_LEN), eb, "sv upload")

    def download(self) -> np.ndarray:
        out = np.empty(1 << self._n, dtype=np.complex128)
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_sv_download(self._dptr, out.view(np.float64).ctypes.data_as(L.c_dp),
                                              self._len, int(self._prec), eb, L.ERR_LEN), eb,
                "sv download")
        return out

    def norm_squared(self) -> float:
        eb = L.errbuf()
        v = C.c_double()
        L.check(L.lib().cast_cuda_norm_squared(self._dptr, self._len, int(self._prec), C.byref(v), eb,
                                               L.ERR_LEN), eb, "norm_squared")
        return v.value

    def normalize(self) -> None:
        n2 = self.norm_squared()
        if not n2 > 0.0:
            raise ValueError("cannot normalize the zero statevector")
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_scale(self._dptr, self._len, int(self._prec), 1.0 / np.sqrt(n2), eb,
                                        L.ERR_LEN), eb, "scale")

    def clone_device(self, stream=None) -> "CudaStatevector":
        out = CudaStatevector(self._n, self._prec)
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_memcpy_dtod_async(out._dptr, self._dptr, self.nbytes(), stream, eb,
                                                    L.ERR_LEN), eb, "clone")
        if stream is None:
            L.check(L.lib().cast_cuda_stream_sync(None, eb, L.ERR_LEN), eb, "clone sync")
        return out


@dataclass
class CudaKernel:
    """kernel.rs:29-90: one compiled (descriptor-loaded) gate."""

    qubits: tuple
    n_gate_qubits: int
    precision: CudaPrecision
    ptx: str
    func_name: str
    module: int
    function: int
    ptx_compile_time: float
    jit_compile_time: float


@dataclass
class KernelExecTime:
    kernel_id: int
    n_gate_qubits: int
    gpu_time: float  # seconds


@dataclass
class SyncStats:
    kernels: list = field(default_factory=list)

    def total_gpu_time(self) -> float:
        return sum(k.gpu_time for k in self.kernels)


class CudaKernelManager:
    """Content-deduplicated gate kernels + a launch queue (kernel.rs:705-977).

    ``generate`` runs compile_gate_ptx -> ptx_to_cubin -> cubin_load ->
    module_get_function once per distinct (matrix, qubits, precision);
    ``apply`` only queues; ``sync`` launches the queue on the manager's stream
    (one event pair per launch when ``timing`` is on, kernel.rs:251-304) and
    waits.  Modules stay loaded: a descriptor module holds only its matrix, so
    the reference's 4-slot LRU (kernel.rs:108) has nothing to evict.
    """

    def __init__(self, spec: CudaKernelGenSpec | None = None, timing: bool = True):
        self._spec = spec or CudaKernelGenSpec.f64()
        self._kernels: list[CudaKernel] = []
        self._dedup: dict[bytes, int] = {}
        self._pending: list[tuple[int, int, int]] = []
        self._lock = threading.Lock()
        self._stream = None
        self.timing = timing

    def spec(self) -> CudaKernelGenSpec:
        return self._spec

    def _ensure_stream(self):
        if self._stream is None:
            eb = L.errbuf()
            self._stream = L.check_ptr(L.lib().cast_cuda_stream_create(eb, L.ERR_LEN), eb, "stream")
        return self._stream

    @property
    def stream(self):
        return self._ensure_stream()

    def __del__(self):
        try:
            lib = L.lib()
            for k in self._kernels:
                lib.cast_cuda_module_unload(k.module)
            if self._stream:
                lib.cast_cuda_stream_destroy(self._stream)
        except Exception:
            pass

    def generate(self, gate) -> int:
        mat = np.ascontiguousarray(gate.matrix(), dtype=np.complex128)
        qubits = np.ascontiguousarray(gate.qubits(), dtype=np.uint32)
        key = hashlib.blake2b(
            mat.tobytes() + qubits.tobytes() + bytes([int(self._spec.precision)]), digest_size=16
        ).digest()
        with self._lock:
            if key in self._dedup:
                return self._dedup[key]
        lib = L.lib()
        eb = L.errbuf()
        spec = self._spec.to_c()
        ptx_p, fn_p = C.c_void_p(), C.c_void_p()
        kq, prec = C.c_uint32(), C.c_uint8()
        t0 = time.perf_counter()
        rc = lib.cast_cuda_compile_gate_ptx(
            C.byref(spec), mat.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)), mat.size,
            qubits.ctypes.data_as(L.c_u32p), qubits.size, C.byref(ptx_p), C.byref(fn_p),
            C.byref(kq), C.byref(prec), eb, L.ERR_LEN)
        L.check(rc, eb, "compile_gate_ptx")
        t1 = time.perf_counter()
        ptx = C.string_at(ptx_p.value).decode()
        fname = C.string_at(fn_p.value).decode()
        lib.cast_cuda_str_free(ptx_p)
        lib.cast_cuda_str_free(fn_p)
        blob_p, blob_len = C.c_void_p(), C.c_size_t()
        L.check(lib.cast_cuda_ptx_to_cubin(ptx.encode(), C.byref(blob_p), C.byref(blob_len), eb,
                                           L.ERR_LEN), eb, "ptx_to_cubin")
        blob = C.string_at(blob_p.value, blob_len.value)
        lib.cast_cuda_cubin_free(blob_p)
        t2 = time.perf_counter()
        mod = L.check_ptr(lib.cast_cuda_cubin_load(blob, len(blob), eb, L.ERR_LEN), eb, "cubin_load")
        fn = lib.cast_cuda_module_get_function(mod, fname.encode(), eb, L.ERR_LEN)
        if not fn:
            lib.cast_cuda_module_unload(mod)
            L.check_ptr(fn, eb, "module_get_function")
        k = CudaKernel(tuple(int(q) for q in qubits), kq.value, CudaPrecision(prec.value), ptx, fname,
                       mod, fn, t1 - t0, t2 - t1)
        with self._lock:
            if key in self._dedup:  # raced with another generate of the same gate
                lib.cast_cuda_module_unload(mod)
                return self._dedup[key]
            kid = len(self._kernels)
            self._kernels.append(k)
            self._dedup[key] = kid
        return kid

    def kernel(self, kid: int) -> CudaKernel:
        return self._kernels[kid]

    def n_kernels(self) -> int:
        return len(self._kernels)

    def apply(self, kid: int, sv: CudaStatevector) -> None:
        k = self._kernels[kid]
        if k.precision != sv.precision():
            raise ValueError("kernel and statevector precision differ")
        if max(k.qubits) >= sv.n_qubits():
            raise ValueError("gate acts on a qubit outside the statevector")
        self._pending.append((kid, sv.dptr, sv.n_qubits()))

    def sync(self) -> SyncStats:
        lib = L.lib()
        eb = L.errbuf()
        stream = self._ensure_stream()
        pending, self._pending = self._pending, []
        events = []
        try:
            for kid, dptr, n in pending:
                k = self._kernels[kid]
                ev0 = ev1 = None
                if self.timing:
                    ev0 = L.check_ptr(lib.cast_cuda_event_create(eb, L.ERR_LEN), eb, "event")
                    L.check(lib.cast_cuda_event_record(ev0, stream, eb, L.ERR_LEN), eb, "event")
                L.check(lib.cast_cuda_kernel_launch(k.function, stream, dptr, k.n_gate_qubits, n, eb,
                                                    L.ERR_LEN), eb, f"kernel {kid} launch failed")
                if self.timing:
                    ev1 = L.check_ptr(lib.cast_cuda_event_create(eb, L.ERR_LEN), eb, "event")
                    L.check(lib.cast_cuda_event_record(ev1, stream, eb, L.ERR_LEN), eb, "event")
                    events.append((kid, k.n_gate_qubits, ev0, ev1))
            L.check(lib.cast_cuda_stream_sync(stream, eb, L.ERR_LEN), eb, "stream sync")
            stats = SyncStats()
            ms = C.c_float()
            for kid, kq, e0, e1 in events:
                L.check(lib.cast_cuda_event_elapsed_ms(e0, e1, C.byref(ms), eb, L.ERR_LEN), eb, "elapsed")
                stats.kernels.append(KernelExecTime(kid, kq, ms.value * 1e-3))
            return stats
        finally:
            for _, _, e0, e1 in events:
                lib.cast_cuda_event_destroy(e0)
                lib.cast_cuda_event_destroy(e1)
