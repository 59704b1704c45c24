"""ctypes front end of the CPU parity oracle (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY.  This module checks results: tests/,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it; the product package ``cast_simulator_b200`` never does.

The C file restates the reference simulator's scalar FP64 CPU path
(src/cpu/statevector.rs:469-516 of narix10yc/cast_simulator) together with the
gate algebra it depends on; see the header of oracle.c for every citation.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "build")
_LIB_PATH = os.path.join(_BUILD, "liboracle.so")

# gate kinds of or_named_matrix (order matches oracle.c)
I, X, Y, Z, H, S, T, RX, RY, RZ, U3, CX, CZ, CP, SWAP, CCX = range(16)

_lib = None


def build(force: bool = False) -> str:
    """Compile oracle.c (and the threaded CPU baseline) with the committed Makefile."""
    stale = False
    for lib_name, src in (("liboracle.so", "oracle.c"), ("libcpu_baseline.so", "cpu_baseline.cpp")):
        lib_path = os.path.join(_BUILD, lib_name)
        if not os.path.exists(lib_path) or (
                os.path.getmtime(lib_path) < os.path.getmtime(os.path.join(_HERE, src))):
            stale = True
    if force or stale:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _Gate(C.Structure):
    _fields_ = [("k", C.c_uint32), ("qubits", C.c_uint32 * 3), ("mat", C.c_double * 128)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        up = C.POINTER(C.c_uint32)
        L.or_named_matrix.argtypes = [C.c_int, dp, dp]
        L.or_named_matrix.restype = C.c_int
        L.or_canonicalize.argtypes = [dp, up, C.c_uint32]
        L.or_canonicalize.restype = C.c_int
        L.or_matmul.argtypes = [dp, up, C.c_uint32, dp, up, C.c_uint32, dp, up]
        L.or_matmul.restype = C.c_int
        L.or_superop_accumulate.argtypes = [dp, C.c_uint32, C.c_double, dp]
        L.or_apply_gate.argtypes = [dp, C.c_uint32, dp, up, C.c_uint32]
        L.or_apply_gate.restype = C.c_int
        L.or_pdep.argtypes = [C.c_uint64, C.c_uint64]
        L.or_pdep.restype = C.c_uint64
        L.or_snap_matrix.argtypes = [dp, C.c_uint32, C.c_double, C.c_double, C.c_int]
        L.or_seeded_state.argtypes = [dp, C.c_uint32]
        L.or_random_state.argtypes = [dp, C.c_uint32, C.c_uint64]
        L.or_inner.argtypes = [dp, dp, C.c_uint64, dp, dp]
        gp = C.POINTER(_Gate)
        for name in ("or_build_qft_cx",):
            getattr(L, name).argtypes = [C.c_uint32, gp, C.c_uint32]
            getattr(L, name).restype = C.c_uint32
        L.or_build_qft_cp.argtypes = [C.c_uint32, C.c_int, gp, C.c_uint32]
        L.or_build_qft_cp.restype = C.c_uint32
        L.or_build_brickwork.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, gp, C.c_uint32]
        L.or_build_brickwork.restype = C.c_uint32
        L.or_dm_apply_channel.argtypes = [dp, C.c_uint32, dp, dp, C.c_uint32, up, C.c_uint32]
        L.or_dm_apply_channel.restype = C.c_int
        L.or_dm_populations.argtypes = [dp, C.c_uint32, dp]
        L.or_splitmix64.argtypes = [C.POINTER(C.c_uint64)]
        L.or_splitmix64.restype = C.c_uint64
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _up(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _cplx_view(a: np.ndarray) -> np.ndarray:
    """float64 view of a C-contiguous complex128 array (shares memory)."""
    assert a.dtype == np.complex128 and a.flags.c_contiguous
    return a.view(np.float64)


def named(kind: int, *params: float) -> np.ndarray:
    p = np.zeros(3)
    p[: len(params)] = params
    out = np.zeros(2 * 64)
    k = lib().or_named_matrix(kind, _dp(p), _dp(out))
    if k < 0:
        raise ValueError(f"unknown gate kind {kind}")
    d = 1 << k
    return out[: 2 * d * d].view(np.complex128).reshape(d, d).copy()


def canonicalize(mat: np.ndarray, qubits) -> tuple[np.ndarray, tuple[int, ...]]:
    m = np.ascontiguousarray(mat, dtype=np.complex128).copy()
    q = np.ascontiguousarray(qubits, dtype=np.uint32).copy()
    if m.shape != (1 << len(q), 1 << len(q)):
        raise ValueError("matrix dimension does not match number of target qubits")
    rc = lib().or_canonicalize(_dp(_cplx_view(m)), _up(q), len(q))
    if rc == -1:
        raise ValueError("gate qubits must be distinct")
    return m, tuple(int(x) for x in q)


def matmul(a, b):
    """(mat, qubits) of a·b on the union of qubits (b applied first): gate.rs:280-284."""
    ma, qa = a
    mb, qb = b
    ma = np.ascontiguousarray(ma, dtype=np.complex128)
    mb = np.ascontiguousarray(mb, dtype=np.complex128)
    qa = np.ascontiguousarray(qa, dtype=np.uint32)
    qb = np.ascontiguousarray(qb, dtype=np.uint32)
    uk = len(set(qa.tolist()) | set(qb.tolist()))
    out = np.zeros((1 << uk, 1 << uk), dtype=np.complex128)
    qo = np.zeros(uk, dtype=np.uint32)
    rc = lib().or_matmul(_dp(_cplx_view(ma)), _up(qa), len(qa), _dp(_cplx_view(mb)), _up(qb),
                         len(qb), _dp(_cplx_view(out)), _up(qo))
    assert rc == uk
    return out, tuple(int(x) for x in qo)


def pdep(src: int, mask: int) -> int:
    return int(lib().or_pdep(src, mask))


def snap(mat: np.ndarray, ztol: float, otol: float, f32: bool = False) -> np.ndarray:
    m = np.ascontiguousarray(mat, dtype=np.complex128).copy()
    k = int(m.shape[0]).bit_length() - 1
    lib().or_snap_matrix(_dp(_cplx_view(m)), k, ztol, otol, int(f32))
    return m


def apply_gate(sv: np.ndarray, mat: np.ndarray, qubits) -> None:
    """In-place scalar application (cpu/statevector.rs:469-516)."""
    n = int(sv.shape[0]).bit_length() - 1
    m = np.ascontiguousarray(mat, dtype=np.complex128)
    q = np.ascontiguousarray(qubits, dtype=np.uint32)
    rc = lib().or_apply_gate(_dp(_cplx_view(sv)), n, _dp(_cplx_view(m)), _up(q), len(q))
    if rc != 0:
        raise ValueError("invalid gate for statevector")


def seeded_state(n: int) -> np.ndarray:
    sv = np.zeros(1 << n, dtype=np.complex128)
    lib().or_seeded_state(_dp(_cplx_view(sv)), n)
    return sv


def random_state(n: int, seed: int) -> np.ndarray:
    sv = np.zeros(1 << n, dtype=np.complex128)
    lib().or_random_state(_dp(_cplx_view(sv)), n, seed)
    return sv


def zero_state(n: int) -> np.ndarray:
    sv = np.zeros(1 << n, dtype=np.complex128)
    sv[0] = 1.0
    return sv


def _gates_from(buf, count):
    out = []
    for i in range(count):
        g = buf[i]
        d = 1 << g.k
        m = np.frombuffer(g.mat, dtype=np.float64)[: 2 * d * d].view(np.complex128).reshape(d, d)
        out.append((m.copy(), tuple(int(g.qubits[j]) for j in range(g.k))))
    return out


def _build(fn, *args):
    n = fn(*args, None, 0)
    buf = (_Gate * max(n, 1))()
    n2 = fn(*args, buf, n)
    assert n2 == n
    return _gates_from(buf, n)


def qft_cx(n: int):
    return _build(lib().or_build_qft_cx, n)


def qft_cp(n: int, swap: bool = True):
    return _build(lib().or_build_qft_cp, n, int(swap))


def brickwork(n: int, depth: int, seed: int):
    return _build(lib().or_build_brickwork, n, depth, seed)


def simulate(n: int, gates, init: np.ndarray | None = None) -> np.ndarray:
    sv = zero_state(n) if init is None else np.array(init, dtype=np.complex128, copy=True)
    for m, q in gates:
        apply_gate(sv, m, q)
    return sv


def inner(a: np.ndarray, b: np.ndarray) -> complex:
    re = C.c_double()
    im = C.c_double()
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    lib().or_inner(_dp(_cplx_view(a)), _dp(_cplx_view(b)), a.shape[0], C.byref(re), C.byref(im))
    return complex(re.value, im.value)


def fidelity_report(ref: np.ndarray, got: np.ndarray) -> dict:
    """1-|<ref|got>| (the form every result reports), 1-|<ref|got>|^2 (the reference's
    fidelity, cpu/statevector.rs:363-374) and the max amplitude error."""
    ov = inner(ref, got)
    return {
        "one_minus_abs_overlap": 1.0 - abs(ov),
        "one_minus_fidelity_sq": 1.0 - abs(ov) ** 2,
        "max_abs_err": float(np.max(np.abs(np.asarray(ref) - np.asarray(got)))) if len(ref) else 0.0,
    }


def dm_zero(n: int) -> np.ndarray:
    rho = np.zeros(1 << (2 * n), dtype=np.complex128)
    rho[0] = 1.0
    return rho


def dm_apply_channel(rho: np.ndarray, n: int, kraus, weights, qubits) -> None:
    """rho <- sum_b w_b K_b rho K_b^dagger via the superoperator lifting of
    gate.rs:236-257 (qubits ascending, kraus in the gate's local basis)."""
    k = len(qubits)
    d = 1 << k
    ks = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.complex128).reshape(d, d) for x in kraus]))
    w = np.ascontiguousarray(weights, dtype=np.float64)
    q = np.ascontiguousarray(qubits, dtype=np.uint32)
    rc = lib().or_dm_apply_channel(_dp(_cplx_view(rho)), n, _dp(_cplx_view(ks)), _dp(w), len(w),
                                   _up(q), k)
    if rc != 0:
        raise ValueError("invalid channel")


def dm_populations(rho: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros(1 << n)
    lib().or_dm_populations(_dp(_cplx_view(rho)), n, _dp(out))
    return out


class ThreadedState:
    """A statevector held by the threaded split-layout CPU restatement
    (cpu_baseline.cpp, FP64 with CAST's CPU zero/+-1 semantics): the oracle for
    sizes the scalar one cannot finish in seconds (a 30-qubit complex128 state
    is 16 GiB of host memory).  Use as a context manager; ``apply`` runs a gate
    list from |0...0> on `threads` host threads, ``chunk`` reads amplitudes
    [first, first + count) as complex128."""

    def __init__(self, n: int, threads: int | None = None):
        build()
        lib = C.CDLL(os.path.join(_BUILD, "libcpu_baseline.so"))
        lib.cb_alloc.restype = C.c_void_p
        lib.cb_alloc.argtypes = [C.c_uint32, C.c_int]
        lib.cb_free.argtypes = [C.c_void_p]
        lib.cb_zero.argtypes = [C.c_void_p]
        lib.cb_apply.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.c_uint32,
                                 C.c_int]
        lib.cb_apply.restype = C.c_int
        lib.cb_store_range.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_double)]
        lib.cb_store_range.restype = C.c_int
        self._lib, self.n = lib, n
        self.threads = threads or os.cpu_count() or 1
        self._p = lib.cb_alloc(n, 0)
        if not self._p:
            raise MemoryError(f"cannot allocate a {n}-qubit state on the host")
        lib.cb_zero(self._p)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        if self._p:
            self._lib.cb_free(self._p)
            self._p = None

    def apply(self, gates) -> None:
        for m, q in gates:
            mm = np.ascontiguousarray(m, dtype=np.complex128).view(np.float64)
            qq = np.ascontiguousarray(q, dtype=np.uint32)
            if self._lib.cb_apply(self._p, mm.ctypes.data_as(C.POINTER(C.c_double)),
                                  qq.ctypes.data_as(C.POINTER(C.c_uint32)), qq.size, self.threads):
                raise ValueError(f"cb_apply rejected qubits {tuple(q)}")

    def chunk(self, first: int, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.complex128)
        if self._lib.cb_store_range(self._p, first, count,
                                    out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))):
            raise IndexError("amplitude range out of bounds")
        return out


# ── shot sampling (src/simulator/measure.rs:49-76) ──────────────────────────


def compress_bits(idx: np.ndarray, measured) -> np.ndarray:
    """Bits of each index at the measured qubits packed into bits 0..m-1
    (compress_bits in the reference's src/types/mod.rs)."""
    idx = np.asarray(idx, dtype=np.uint64)
    out = np.zeros_like(idx)
    for j, q in enumerate(measured):
        out |= ((idx >> np.uint64(q)) & np.uint64(1)) << np.uint64(j)
    return out


def batch_sample_fp64(probs: np.ndarray, u: np.ndarray) -> np.ndarray:
    """The reference's inverse-CDF rule (measure.rs:61-75): cdf = running FP64
    sum of the probabilities in index order; the outcome of u is the first index
    whose cdf entry is > u, clamped to the last index."""
    cdf = np.cumsum(np.asarray(probs, dtype=np.float64))
    return np.minimum(np.searchsorted(cdf, np.asarray(u, dtype=np.float64), side="right"),
                      cdf.size - 1).astype(np.uint64)


def sample_fixed_point(psi: np.ndarray, u: np.ndarray, scale: float = 2.0 ** 62) -> np.ndarray:
    """The same rule over the 64-bit fixed-point CDF the device uses: p_i =
    re^2 + im^2 (separately rounded), q_i = round-half-even(p_i * scale) as
    uint64, exact prefix sums, target t = floor(u * float(Q)) with Q the integer
    total, outcome = first index whose inclusive prefix is > t (the last index
    if none).  scale = 2^62 is the device's choice for a state whose total
    probability lies in (0.5, 2)."""
    psi = np.asarray(psi, dtype=np.complex128)
    p = psi.real * psi.real + psi.imag * psi.imag
    q = np.rint(p * scale).astype(np.uint64)
    cdf = np.cumsum(q, dtype=np.uint64)
    t = np.floor(np.asarray(u, dtype=np.float64) * float(cdf[-1])).astype(np.uint64)
    return np.minimum(np.searchsorted(cdf, t, side="right"), cdf.size - 1).astype(np.uint64)
