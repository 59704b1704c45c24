"""The allocation-free norm^2 entry point (cast_b200_norm_squared_noalloc).

It exists for callers that cannot let the library allocate device memory: a
host whose device memory is owned by a pool or arena that accounts for every
byte, or a service that forbids allocations once running (cudaMalloc and
cudaFree may synchronise the whole device).  Its scratch is a fixed array
inside the library.  These tests call it through
the C ABI and check it against the allocating cast_cuda_norm_squared on two
calls in a row (the shared array keeps the previous call's contents), and that
an input larger than its fixed scratch supports is refused with an error.
This file is collected last so that a failure here stops a -x run only after
every other test has run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # FP64 accumulation in both entry points; only the summation order differs


def _norms(lib, L, sv):
    eb = L.errbuf()
    ref = C.c_double()
    L.check(lib.cast_cuda_norm_squared(sv.dptr, len(sv), int(sv.precision()), C.byref(ref), eb,
                                       L.ERR_LEN), eb, "norm_squared")
    got = C.c_double()
    rc = lib.cast_b200_norm_squared_noalloc(sv.dptr, len(sv), int(sv.precision()), C.byref(got),
                                            None, eb, L.ERR_LEN)
    assert rc == 0, eb.value
    assert eb.value == b""
    return ref.value, got.value


@pytest.mark.parametrize("prec", [1, 0])
def test_noalloc_matches_allocating_norm_twice(cblib, prec):
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu

    rng = np.random.default_rng(77 + prec)
    # two calls in a row on different inputs: the second must not see the first's partials
    for n, scale in ((20, 3.0), (13, 0.5)):
        sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
        amps = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)) * scale
        sv.upload(amps)
        ref, got = _norms(cblib, L, sv)
        assert abs(got - ref) <= REL_TOL * ref, (n, ref, got)
        stored = sv.download()
        assert abs(got - float(np.sum(np.abs(stored) ** 2))) <= 1e-10 * ref


@pytest.mark.parametrize("prec", [1, 0])
def test_noalloc_ragged_counts(cblib, prec):
    """Counts that are not a multiple of the 16-byte vector width (the scalar
    tail) and counts whose last block is partial, on one buffer, against numpy
    over the same leading scalars of the downloaded statevector."""
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu

    n = 17
    sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    rng = np.random.default_rng(5 + prec)
    sv.upload(rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n))
    scalars = sv.download().view(np.float64)
    if prec == 0:
        scalars = scalars.astype(np.float32).astype(np.float64)
    per_vec = 2 if prec == 1 else 4
    per_block = 256 * 64 * per_vec  # scalars one first-pass block covers
    full = len(sv)
    counts = [full - 1, full - 3, 3 * per_block + 5 * per_vec + 1, per_block - 1, 1, 0]
    eb = L.errbuf()
    for count in counts:
        got = C.c_double(-1.0)
        rc = cblib.cast_b200_norm_squared_noalloc(sv.dptr, count, prec, C.byref(got), None, eb,
                                                  L.ERR_LEN)
        assert rc == 0, eb.value
        want = float(np.sum(scalars[:count] ** 2))
        assert abs(got.value - want) <= 1e-12 * max(want, 1.0), (count, got.value, want)


def test_noalloc_rejects_inputs_beyond_its_scratch(cblib):
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu

    sv = cu.CudaStatevector(4, cu.CudaPrecision.F64)
    sv.zero()
    eb = L.errbuf()
    out = C.c_double(-1.0)
    too_many = (1 << 32) + 2  # F64 limit is 2^32 scalars; rejected before any launch
    rc = cblib.cast_b200_norm_squared_noalloc(sv.dptr, too_many, 1, C.byref(out), None, eb, L.ERR_LEN)
    assert rc == 1 and b"exceed the maximum" in eb.value and out.value == -1.0
    rc = cblib.cast_b200_norm_squared_noalloc(0, 8, 1, C.byref(out), None, eb, L.ERR_LEN)
    assert rc == 1 and b"must not be null" in eb.value
    rc = cblib.cast_b200_norm_squared_noalloc(sv.dptr + 8, 8, 1, C.byref(out), None, eb, L.ERR_LEN)
    assert rc == 1 and b"16-byte aligned" in eb.value and out.value == -1.0
