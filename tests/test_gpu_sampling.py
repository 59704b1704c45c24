"""On-device shot sampling (cast_b200_sample / cast_b200_sample_at) against the
oracle: the reference draws shots by the inverse CDF on the host after
downloading the statevector (src/simulator/measure.rs:49-76,
src/simulator/mod.rs:282-291).  With the caller's uniforms the device must give
exactly the oracle's indices over the same fixed-point CDF, and the reference's
FP64 rule wherever a target is not within rounding of a CDF boundary; with the
device's own draws the counts must pass a chi-square test against the oracle's
probabilities."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import cuda, simulator

    return cuda, simulator


def _upload(cu, psi, prec):
    sv = cu.CudaStatevector(int(np.log2(psi.size)), cu.CudaPrecision(prec))
    sv.upload(psi)
    return sv, sv.download()  # the amplitudes the device holds


@pytest.mark.parametrize("n", [1, 5, 12, 17])
@pytest.mark.parametrize("prec", [1, 0])
def test_given_uniforms_match_the_oracle_exactly(mods, oracle, n, prec):
    cu, S = mods
    sv, held = _upload(cu, oracle.random_state(n, 40 + n), prec)
    rng = np.random.default_rng(n)
    u = np.sort(np.concatenate([[0.0, 1.0 - 2.0 ** -53], rng.random(4000)]))
    got = S.sample(sv, u.size, uniforms=u)
    want = oracle.sample_fixed_point(held, u)
    assert np.array_equal(got, want)
    assert np.all(np.diff(got.astype(np.int64)) >= 0)  # ascending sampled index
    if prec == 1:
        # the reference's FP64 CDF gives the same outcomes (no target lands within
        # rounding of a boundary for these draws)
        p = np.abs(held) ** 2
        ref = oracle.batch_sample_fp64(p, u * p.sum())
        assert np.array_equal(got, ref)


def test_measured_subset_keys(mods, oracle):
    cu, S = mods
    n, measured = 14, [13, 2, 7, 0]
    sv, held = _upload(cu, oracle.random_state(n, 9), 1)
    u = np.sort(np.random.default_rng(2).random(3000))
    got = S.sample(sv, u.size, measured=measured, uniforms=u)
    want = oracle.compress_bits(oracle.sample_fixed_point(held, u), measured)
    assert np.array_equal(got, want)
    assert got.max() < 16


@pytest.mark.parametrize("n,measured,shots", [(12, None, 400_000), (20, list(range(0, 20, 2)), 300_000)])
def test_seeded_counts_pass_chi_square(mods, oracle, n, measured, shots):
    from scipy import stats

    cu, S = mods
    sv, held = _upload(cu, oracle.random_state(n, 77), 1)
    p = np.abs(held) ** 2
    p /= p.sum()
    if measured is not None:
        keys = oracle.compress_bits(np.arange(p.size), measured).astype(np.int64)
        p = np.bincount(keys, weights=p, minlength=1 << len(measured))
    hist = S.sample_histogram(sv, shots, seed=123, measured=measured)
    counts = np.zeros(p.size)
    for k, c in hist.items():
        counts[k] = c
    assert counts.sum() == shots
    exp = p * shots
    big = exp >= 5
    obs_b = np.append(counts[big], counts[~big].sum())
    exp_b = np.append(exp[big], exp[~big].sum())
    if exp_b[-1] == 0:
        obs_b, exp_b = obs_b[:-1], exp_b[:-1]
    chi2 = float(np.sum((obs_b - exp_b) ** 2 / exp_b))
    pval = stats.chi2.sf(chi2, obs_b.size - 1)
    assert pval > 1e-6, (chi2, obs_b.size, pval)


def test_seed_determinism(mods, oracle):
    cu, S = mods
    sv, _ = _upload(cu, oracle.random_state(16, 5), 0)
    a = S.sample(sv, 20000, seed=7)
    b = S.sample(sv, 20000, seed=7)
    c = S.sample(sv, 20000, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.all(np.diff(a.astype(np.int64)) >= 0)


def test_edge_cases(mods, oracle):
    from cast_simulator_b200 import _lib as L

    cu, S = mods
    n = 9
    # a basis state: every shot gives it; zero-probability amplitudes are never drawn
    psi = np.zeros(1 << n, dtype=complex)
    psi[300] = 1j
    sv, _ = _upload(cu, psi, 1)
    assert set(S.sample(sv, 5000, seed=1).tolist()) == {300}
    psi = np.zeros(1 << n, dtype=complex)
    psi[[3, 17, 400]] = [0.6, 0.0, 0.8]
    sv, _ = _upload(cu, psi, 0)
    keys = set(S.sample(sv, 20000, seed=2).tolist())
    assert keys == {3, 400}
    assert S.sample(sv, 0).size == 0
    # an unnormalised state samples its normalised distribution
    big, _ = _upload(cu, oracle.random_state(n, 3) * 5.0, 1)
    small, _ = _upload(cu, oracle.random_state(n, 3) * 1e-4, 1)
    ref, _ = _upload(cu, oracle.random_state(n, 3), 1)
    u = np.sort(np.random.default_rng(4).random(5000))
    r = S.sample(ref, u.size, uniforms=u)
    for other in (big, small):
        assert np.mean(S.sample(other, u.size, uniforms=u) == r) > 0.999
    # errors: zero state, bad measured list, unsorted or out-of-range uniforms
    zero = cu.CudaStatevector(n, cu.CudaPrecision.F64)
    zero.upload(np.zeros(1 << n, dtype=complex))
    with pytest.raises(L.CudaError, match="zero"):
        S.sample(zero, 10, seed=1)
    with pytest.raises(L.CudaError, match="distinct"):
        S.sample(ref, 10, seed=1, measured=[1, 1])
    with pytest.raises(L.CudaError, match="non-decreasing"):
        S.sample(ref, 3, uniforms=[0.5, 0.2, 0.9])
    with pytest.raises(L.CudaError, match="non-decreasing"):
        S.sample(ref, 2, uniforms=[0.5, 1.0])


def test_caller_output_buffer(mods, oracle):
    """Keys written into a caller's buffer (reused across calls, page-locked or
    not) equal those of a fresh array; a buffer of the wrong type or size is
    refused before the device is touched."""
    import torch

    cu, S = mods
    sv, _ = _upload(cu, oracle.random_state(14, 8), 1)
    fresh = S.sample(sv, 30000, seed=5)
    pinned = torch.empty(30000, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    plain = np.zeros(30000, dtype=np.uint64)
    for buf in (pinned, plain, pinned):
        got = S.sample(sv, 30000, seed=5, out=buf)
        assert got is buf
        assert np.array_equal(got, fresh)
    with pytest.raises(ValueError):
        S.sample(sv, 30000, seed=5, out=np.zeros(30000, dtype=np.int32))
    with pytest.raises(ValueError):
        S.sample(sv, 30000, seed=5, out=np.zeros(100, dtype=np.uint64))


def test_concurrent_callers_get_their_own_scratch(mods, oracle):
    """Threads sampling at the same time on their own streams each take a
    scratch buffer of their own from the cache: every result equals the same
    draw made alone, and repeated rounds reuse the buffers."""
    import threading

    cu, S = mods
    svs = [_upload(cu, oracle.random_state(15, 20 + i), i % 2)[0] for i in range(4)]
    alone = [S.sample(sv, 20000 + 1000 * i, seed=7 + i) for i, sv in enumerate(svs)]
    for _ in range(3):
        got = [None] * 4
        errors = []

        def run(i):
            try:
                st = S.Stream()
                got[i] = S.sample(svs[i], 20000 + 1000 * i, seed=7 + i, stream=st)
            except Exception as e:  # reported below
                errors.append(e)

        threads = [threading.Thread(target=run, args=(i,)) for i in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors
        for a, g in zip(alone, got):
            assert np.array_equal(a, g)


def test_quantum_state_sample_histogram(mods, oracle):
    """QuantumState.sample on a simulated circuit: H on qubit 0 and CX(0, 3) give
    outcomes 0b0000 and 0b1001 only, in roughly equal counts."""
    from cast_simulator_b200.fusion import CircuitGraph
    from cast_simulator_b200.simulator import Simulator
    from cast_simulator_b200.types import QuantumCircuit, QuantumGate

    circ = QuantumCircuit(4)
    circ.add(QuantumGate.h(0))
    circ.add(QuantumGate.cx(0, 3))
    st = Simulator.f64().simulate(CircuitGraph.from_circuit(circ))
    hist = st.sample(10000, seed=3)
    assert set(hist) == {0, 9} and abs(hist[0] - 5000) < 300
    hist2 = st.sample(10000, measured=[3], seed=3)
    assert set(hist2) == {0, 1}
