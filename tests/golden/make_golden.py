"""Generate golden vectors from the reference's own QASM fixture.

Run in a container where the reference checkout is mounted:

    python tests/golden/make_golden.py <path to the reference checkout>

It reads ``tests/assets/qft_14.qasm`` of narix10yc/cast_simulator (the QFT with
each controlled phase decomposed into CX + u3 phases, qft_14.qasm:3-8), runs it
through a small numpy interpreter written from the OpenQASM 2.0 definitions of
h / u3 / cx / swap (independent of the oracle's C code), and stores

  * qft14_seeded.npy  - final amplitudes for the reference test input
                        amp_i ~ (i+1, 0.5 i - 0.25), normalised
                        (tests/cpu_cuda_compare.rs:54-69);
  * qft14_meta.json   - gate counts and the fixture's sha256.

Only the derived vectors are committed, never the fixture text itself.
The oracle's QFT-CX builder and gate semantics are pinned against these files
by tests/test_oracle.py.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _angle(expr: str) -> float:
    expr = expr.strip()
    if not re.fullmatch(r"[0-9pi+\-*/. ()]+", expr):
        raise ValueError(f"unsupported angle expression {expr!r}")
    return float(eval(expr, {"__builtins__": {}}, {"pi": math.pi}))


def _apply_1q(psi: np.ndarray, n: int, q: int, m: np.ndarray) -> np.ndarray:
    t = psi.reshape((2,) * n)
    ax = n - 1 - q  # C-order reshape: axis 0 is the most significant bit
    t = np.moveaxis(np.tensordot(m, t, axes=([1], [ax])), 0, ax)
    return t.reshape(-1)


def _apply_cx(psi: np.ndarray, n: int, c: int, tq: int) -> np.ndarray:
    idx = np.arange(psi.shape[0])
    sel = ((idx >> c) & 1) == 1
    out = psi.copy()
    out[sel] = psi[idx[sel] ^ (1 << tq)]
    return out


def _apply_swap(psi: np.ndarray, n: int, a: int, b: int) -> np.ndarray:
    idx = np.arange(psi.shape[0])
    ba = (idx >> a) & 1
    bb = (idx >> b) & 1
    src = idx ^ ((ba ^ bb) << a) ^ ((ba ^ bb) << b)
    return psi[src]


def run_qasm(text: str, psi: np.ndarray) -> tuple[np.ndarray, dict]:
    n = None
    counts: dict[str, int] = {}
    for raw in text.splitlines():
        line = raw.split("//")[0].strip()
        if not line or line.startswith("OPENQASM") or line.startswith("include"):
            continue
        line = line.rstrip(";").strip()
        m = re.fullmatch(r"qreg\s+q\[(\d+)\]", line)
        if m:
            n = int(m.group(1))
            assert psi.shape[0] == 1 << n
            continue
        m = re.fullmatch(r"(\w+)(?:\(([^)]*)\))?\s+(.*)", line)
        if not m:
            raise ValueError(f"cannot parse {raw!r}")
        name, params, args = m.group(1), m.group(2), m.group(3)
        qs = [int(x) for x in re.findall(r"q\[(\d+)\]", args)]
        counts[name] = counts.get(name, 0) + 1
        if name == "h":
            s = 1.0 / math.sqrt(2.0)
            psi = _apply_1q(psi, n, qs[0], np.array([[s, s], [s, -s]], dtype=complex))
        elif name == "u3":
            th, ph, la = (_angle(p) for p in params.split(","))
            c, s = math.cos(th / 2), math.sin(th / 2)
            mat = np.array(
                [[c, -np.exp(1j * la) * s], [np.exp(1j * ph) * s, np.exp(1j * (ph + la)) * c]],
                dtype=complex,
            )
            psi = _apply_1q(psi, n, qs[0], mat)
        elif name == "cx":
            psi = _apply_cx(psi, n, qs[0], qs[1])
        elif name == "swap":
            psi = _apply_swap(psi, n, qs[0], qs[1])
        else:
            raise ValueError(f"gate {name} not used by the fixture")
    return psi, {"n_qubits": n, "gate_counts": counts}


def seeded_state(n: int) -> np.ndarray:
    i = np.arange(1 << n, dtype=np.float64)
    v = (i + 1.0) + 1j * (0.5 * i - 0.25)
    return v / np.linalg.norm(v)


def main(ref_root: str) -> None:
    path = os.path.join(ref_root, "tests", "assets", "qft_14.qasm")
    with open(path, "rb") as f:
        raw = f.read()
    text = raw.decode()
    out, meta = run_qasm(text, seeded_state(14))
    np.save(os.path.join(HERE, "qft14_seeded.npy"), out.astype(np.complex128))
    zero = np.zeros(1 << 14, dtype=complex)
    zero[0] = 1
    z_out, _ = run_qasm(text, zero)
    meta["sha256"] = hashlib.sha256(raw).hexdigest()
    meta["source"] = "narix10yc/cast_simulator tests/assets/qft_14.qasm"
    meta["input"] = "amp_i ~ (i+1, 0.5 i - 0.25), normalised (tests/cpu_cuda_compare.rs:54-69)"
    meta["zero_state_max_dev_from_uniform"] = float(np.max(np.abs(np.abs(z_out) - 2.0**-7)))
    with open(os.path.join(HERE, "qft14_meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print(json.dumps(meta, indent=1, sort_keys=True))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
