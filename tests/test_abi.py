"""The C-ABI library: loads, exports every declared symbol, and the
GPU-free parts of the gate pipeline (descriptor + blob) behave like the
reference's (error convention of src/cpp/internal/err_buf.hpp:12-23)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        names |= set(re.findall(r"\b(cast_\w+)\s*\(", text))
    return sorted(names)


def test_exports_every_declared_symbol(cblib):
    names = declared_symbols()
    assert len(names) >= 26
    missing = [n for n in names if not hasattr(cblib, n)]
    assert not missing, missing


def _compile(cblib, mat, qubits, prec=1, ztol=1e-12, otol=1e-12):
    from cast_simulator_b200 import _lib as L

    spec = L.KernelGenSpec(prec, ztol, otol, 10, 0, 128)
    m = np.ascontiguousarray(mat, dtype=np.complex128)
    q = np.ascontiguousarray(qubits, dtype=np.uint32)
    ptx, fn = C.c_void_p(), C.c_void_p()
    kq, pr = C.c_uint32(), C.c_uint8()
    eb = L.errbuf()
    rc = cblib.cast_cuda_compile_gate_ptx(
        C.byref(spec), m.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)), m.size,
        q.ctypes.data_as(L.c_u32p), q.size, C.byref(ptx), C.byref(fn), C.byref(kq), C.byref(pr),
        eb, L.ERR_LEN)
    return rc, eb.value.decode(), ptx, fn, kq.value, pr.value


def test_compile_descriptor_roundtrip(cblib):
    rng = np.random.default_rng(1)
    m = rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8))
    m[0, 0] = 1 + 1e-14  # snapped to exactly 1 (otol / K)
    rc, err, ptx, fn, k, pr = _compile(cblib, m, [1, 4, 9])
    assert rc == 0 and err == "" and k == 3 and pr == 1
    text = C.string_at(ptx.value).decode()
    assert C.string_at(fn.value) == b"k_gate"
    assert ".qubits 1 4 9" in text and ".precision f64" in text
    from cast_simulator_b200 import _lib as L

    blob, ln = C.c_void_p(), C.c_size_t()
    eb = L.errbuf()
    assert cblib.cast_cuda_ptx_to_cubin(text.encode(), C.byref(blob), C.byref(ln), eb, L.ERR_LEN) == 0
    raw = C.string_at(blob.value, ln.value)
    vals = np.frombuffer(raw[-64 * 16:], dtype=np.complex128).reshape(8, 8)
    assert vals[0, 0] == 1.0 and np.array_equal(vals[1:], m[1:])
    cblib.cast_cuda_cubin_free(blob)
    cblib.cast_cuda_str_free(ptx)
    cblib.cast_cuda_str_free(fn)


def test_compile_errors(cblib):
    rc, err, *_ = _compile(cblib, np.eye(4), [0])
    assert rc == 1 and "matrixLen" in err
    rc, err, *_ = _compile(cblib, np.eye(4), [3, 1])
    assert rc == 1 and "ascending" in err
    rc, err, *_ = _compile(cblib, np.eye(256), list(range(8)))
    assert rc == 1 and "not supported" in err
    rc, err, *_ = _compile(cblib, np.eye(2), [0], prec=5)
    assert rc == 1 and "precision" in err


def test_bad_descriptor_rejected(cblib):
    from cast_simulator_b200 import _lib as L

    blob, ln = C.c_void_p(), C.c_size_t()
    eb = L.errbuf()
    assert cblib.cast_cuda_ptx_to_cubin(b".version 8.0\n", C.byref(blob), C.byref(ln), eb, L.ERR_LEN) == 1
    assert b"descriptor" in eb.value
    assert cblib.cast_cuda_cubin_load(b"garbage-garbage-garbage-garbage-" * 4, 128, eb, L.ERR_LEN) is None
    assert b"not a cast_b200 gate module" in eb.value
    assert cblib.cast_cuda_kernel_launch(None, None, 0, 1, 4, eb, L.ERR_LEN) == 1
    assert b"must not be null" in eb.value


def test_truncated_blob_rejected_before_any_read(cblib):
    """cubin_load never reads past the length it is given: a length of 0, one
    shorter than the header, and one that cuts the matrix short are refused
    (these return before the device is touched, so they run without a GPU)."""
    from cast_simulator_b200 import _lib as L

    rc, _, ptx, fn, *_ = _compile(cblib, np.eye(4), [0, 1])
    assert rc == 0
    blob, ln = C.c_void_p(), C.c_size_t()
    eb = L.errbuf()
    assert cblib.cast_cuda_ptx_to_cubin(C.string_at(ptx.value), C.byref(blob), C.byref(ln), eb,
                                        L.ERR_LEN) == 0
    raw = C.string_at(blob.value, ln.value)
    for n in (0, 16, ln.value - 1):
        buf = C.create_string_buffer(raw[:n], max(n, 1))
        eb = L.errbuf()
        assert cblib.cast_cuda_cubin_load(buf, n, eb, L.ERR_LEN) is None
        assert b"truncated" in eb.value, (n, eb.value)
    cblib.cast_cuda_cubin_free(blob)
    cblib.cast_cuda_str_free(ptx)
    cblib.cast_cuda_str_free(fn)


def test_trajectory_threads_setting(cblib):
    """Trajectory programs are built on the host; the launch-shape knob accepts
    512, 1024 and 0 (by state size) threads and any CTA count."""
    from cast_simulator_b200 import _lib as L

    eb = L.errbuf()
    prog = cblib.cast_b200_traj_create(12, eb, L.ERR_LEN)
    assert prog
    try:
        for t in (0, 512, 1024):
            assert cblib.cast_b200_traj_set_launch(prog, t, 0, eb, L.ERR_LEN) == 0
        assert cblib.cast_b200_traj_set_launch(prog, 512, 100, eb, L.ERR_LEN) == 0
        for t in (256, 384, 2048):
            assert cblib.cast_b200_traj_set_launch(prog, t, 0, eb, L.ERR_LEN) == 1
            assert b"512, 1024 or 0" in eb.value
        assert cblib.cast_b200_traj_set_launch(None, 512, 0, eb, L.ERR_LEN) == 1
    finally:
        cblib.cast_b200_traj_destroy(prog)


def test_gate_engine_routing(cblib):
    """Kernel routing is a pure host decision, the same one a launch takes: dense
    gates by width and low targets, sparse gates (at most 2^k / 4 nonzeros a row,
    k >= 5) on the CSR kernels, split-precision complex64 k = 5, 6 on the tensor
    cores."""
    from cast_simulator_b200.cuda import CudaPrecision as P
    from cast_simulator_b200.simulator import gate_engine

    rng = np.random.default_rng(3)

    def haar(k):
        z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
        return np.linalg.qr(z)[0]

    def mono(k):
        d = 1 << k
        m = np.zeros((d, d), dtype=complex)
        m[np.arange(d), rng.permutation(d)] = 1.0
        return m

    F64, F32 = P.F64, P.F32
    assert gate_engine(haar(4), (16, 17, 18, 19), 20, F64) == "register"
    assert gate_engine(haar(4), (0, 1, 2, 3), 20, F64) == "tile"
    assert gate_engine(haar(4), (0, 1, 2, 3), 10, F64) == "register"  # no 2048-amplitude tile
    assert gate_engine(haar(3), (0, 1, 2), 12, F64) == "tile"          # 4096-amplitude tile
    assert gate_engine(haar(3), (0, 1, 2), 11, F64) == "register"
    assert gate_engine(haar(3), (1, 2, 3), 20, F32) == "tile"
    assert gate_engine(haar(3), (2, 3, 4), 20, F32) == "register"
    assert gate_engine(haar(2), (0, 9), 20, F64) == "register"          # one low target
    assert gate_engine(haar(5), (10, 11, 12, 13, 14), 20, F64) == "register"
    assert gate_engine(haar(6), tuple(range(10, 16)), 20, F64) == "staged"
    assert gate_engine(mono(6), tuple(range(10, 16)), 20, F64) == "sparse"
    assert gate_engine(mono(6), tuple(range(6)), 20, F64) == "sparse_tile"
    assert gate_engine(mono(6), tuple(range(6)), 10, F64) == "sparse"
    assert gate_engine(mono(6), tuple(range(6)), 11, F32) == "sparse"    # FP32 tile: 4096
    assert gate_engine(mono(6), tuple(range(6)), 12, F32) == "sparse_tile"
    assert gate_engine(mono(4), tuple(range(4)), 20, F64) == "tile"      # sparse only from k = 5
    assert gate_engine(haar(6), tuple(range(10, 16)), 20, F32, split_precision=True) == "tensor"
    assert gate_engine(haar(5), (0, 2, 4, 6, 8), 20, F32, split_precision=True) == "tensor"
    assert gate_engine(mono(6), tuple(range(10, 16)), 20, F32, split_precision=True) == "sparse"
    assert gate_engine(haar(6), tuple(range(10, 16)), 20, F64, split_precision=True) == "staged"
    assert gate_engine(haar(4), (0, 1, 2, 3), 20, F32, split_precision=True) == "tile"
    # unsorted qubits are canonicalised like every other entry point
    assert gate_engine(mono(6), (15, 10, 11, 12, 13, 14), 20, F64) == "sparse"
    with pytest.raises(RuntimeError, match="outside"):
        gate_engine(haar(2), (0, 25), 20, F64)


def test_kernel_choice_routing(cblib):
    """Autotuned choices route a low-target class to the register or tile
    kernel, leave other classes and high-target gates alone, and reset to the
    built-in rule; out-of-range classes are refused with a message."""
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200.cuda import CudaPrecision as P
    from cast_simulator_b200.simulator import gate_engine, set_kernel_choice

    rng = np.random.default_rng(4)
    z = rng.standard_normal((16, 16)) + 1j * rng.standard_normal((16, 16))
    m4 = np.linalg.qr(z)[0]
    try:
        set_kernel_choice(P.F64, 4, 0b1111, "register")
        assert gate_engine(m4, (0, 1, 2, 3), 20, P.F64) == "register"
        assert gate_engine(m4, (0, 1, 2, 3), 20, P.F32) == "tile"  # the other precision
        assert gate_engine(m4, (0, 1, 2, 4), 20, P.F64) == "tile"  # another low mask
        set_kernel_choice(P.F32, 4, 0b10100, "tile", 12)
        assert gate_engine(m4, (2, 4, 10, 15), 20, P.F32) == "tile"
        assert gate_engine(m4, (2, 4, 9, 10), 11, P.F32) == "register"  # no 4096-amplitude tile
        assert gate_engine(m4, (10, 11, 12, 15), 20, P.F32) == "register"  # no low target
        set_kernel_choice(P.F64, 4, 0b1111, None)
        assert gate_engine(m4, (0, 1, 2, 3), 20, P.F64) == "tile"
        for bad in [(P.F64, 5, 1, "tile", 0), (P.F64, 2, 0b111, "tile", 0), (P.F64, 2, 0, "tile", 0),
                    (P.F64, 2, 32, "tile", 0), (P.F64, 2, 3, "tile", 10)]:
            with pytest.raises(L.CudaError, match="kernel choice"):
                set_kernel_choice(*bad)
    finally:
        set_kernel_choice(P.F64, 4, 0b1111, None)
        set_kernel_choice(P.F32, 4, 0b10100, None)


def test_kernel_classes_cover_low_masks():
    from cast_simulator_b200.autotune import class_targets, kernel_classes

    cls = kernel_classes()
    assert len(cls) == 5 + 15 + 25 + 30
    for k, mask in cls:
        q = class_targets(26, k, mask)
        assert len(set(q)) == k and list(q) == sorted(q)
        assert sum(1 << b for b in q if b < 5) == mask


def test_compile_is_reentrant(cblib):
    """The reference compiles gates from several worker threads at once
    (cuda/kernel.rs:1078-1096): concurrent calls give exactly the descriptors
    that serial calls give (ctypes drops the GIL around each call)."""
    import threading

    rng = np.random.default_rng(11)
    jobs = []
    for _ in range(160):
        k = int(rng.integers(1, 5))
        q = np.sort(rng.choice(20, size=k, replace=False))
        d = 1 << k
        jobs.append((rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)), q,
                     int(rng.integers(0, 2))))

    def descriptor(job):
        m, q, prec = job
        rc, err, ptx, fn, k, pr = _compile(cblib, m, q, prec)
        assert rc == 0, err
        text = C.string_at(ptx.value)
        cblib.cast_cuda_str_free(ptx)
        cblib.cast_cuda_str_free(fn)
        return text, k, pr

    serial = [descriptor(j) for j in jobs]
    out = [None] * len(jobs)
    errors = []

    def worker(t):
        try:
            for i in range(t, len(jobs), 8):
                out[i] = descriptor(jobs[i])
        except Exception as e:  # reported below, on the test's thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert out == serial


def test_misaligned_pointers_rejected_without_touching_the_device(cblib):
    """Every kernel reads amplitudes as 16-byte vectors, so an interior pointer
    that is not 16-byte aligned is refused with an error instead of reaching a
    kernel.  The check comes before any CUDA call, so this runs without a GPU;
    the fake address is never dereferenced."""
    from cast_simulator_b200 import _lib as L

    bad = 0x10000008
    eb = L.errbuf()
    m = np.ascontiguousarray(np.eye(2, dtype=np.complex128))
    q = np.zeros(1, dtype=np.uint32)
    out = (C.c_double * 64)()
    re, im = C.c_double(), C.c_double()
    calls = [
        lambda: cblib.cast_b200_apply_gate(bad, 4, 1, m.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), q.ctypes.data_as(L.c_u32p), 1, 1e-12, 1e-12, None, eb, L.ERR_LEN),
        lambda: cblib.cast_cuda_norm_squared(bad, 32, 1, out, eb, L.ERR_LEN),
        lambda: cblib.cast_cuda_scale(bad, 32, 0, 2.0, eb, L.ERR_LEN),
        lambda: cblib.cast_b200_inner_product(0x10000000, bad, 4, 1, C.byref(re), C.byref(im), None,
                                              eb, L.ERR_LEN),
        lambda: cblib.cast_b200_qubit_populations(bad, 4, 1, out, None, None, eb, L.ERR_LEN),
        lambda: cblib.cast_b200_marginal_probabilities(bad, 4, 1, q.ctypes.data_as(L.c_u32p), 1, out,
                                                       None, eb, L.ERR_LEN),
        lambda: cblib.cast_b200_dm_populations(bad, 2, 1, out, None, eb, L.ERR_LEN),
        lambda: cblib.cast_b200_norm_squared_noalloc(bad, 32, 1, out, None, eb, L.ERR_LEN),
        lambda: cblib.cast_b200_damping_sums(bad, 4, 1, 3, 0.1, C.byref(re), C.byref(im), None, eb,
                                             L.ERR_LEN),
        lambda: cblib.cast_b200_scale_popc(bad, 4, 0, 3, 0.5, 1.0, None, eb, L.ERR_LEN),
    ]
    for i, call in enumerate(calls):
        eb.value = b""
        assert call() == 1, i
        assert b"16-byte aligned" in eb.value, (i, eb.value)


def test_default_kernel_table_is_well_formed():
    """The built-in routing table in gate_kernels.cu has one 32-entry row per
    precision and k, 'r' / 'a' / 'b' exactly on the masks a k-qubit gate can
    have, and round-trips through the autotuner's emitter."""
    import os
    import re

    from cast_simulator_b200.autotune import cxx_table

    src = open(os.path.join(os.path.dirname(__file__), "..", "cast_simulator_b200", "csrc",
                            "gate_kernels.cu")).read()
    body = src[src.index("kDefaultChoice[2][5][33] = {"):]
    body = body[:body.index("};")]
    rows = re.findall(r'\{""((?:, "[^"]*")*)\}', body)
    assert len(rows) == 2
    table = {}
    recs = []
    for p, row in zip(("f32", "f64"), rows):
        cells = re.findall(r'"([^"]*)"', row)
        assert len(cells) == 4
        for k, cell in zip(range(1, 5), cells):
            assert len(cell) == 32
            for m, ch in enumerate(cell):
                possible = m > 0 and bin(m).count("1") <= k
                assert (ch in "rab") == possible and (ch == "-") == (not possible), (p, k, m, ch)
                if possible:
                    eng, tb = {"r": ("register", 0), "a": ("tile", 11), "b": ("tile", 12)}[ch]
                    recs.append({"precision": p, "k": k, "low_mask": m, "engine": eng, "tile_bits": tb})
            table[(p, k)] = cell
    emitted = cxx_table(recs).splitlines()
    for line, p in zip(emitted, ("f32", "f64")):
        assert line.strip() == "{" + '""' + "".join(f', "{table[(p, k)]}"' for k in range(1, 5)) + "},"
