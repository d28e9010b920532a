"""Seeded circuit generators for the benchmark workloads and the tests.

A circuit is a list of (op, params, targets, negctrls, ctrls) tuples; op is a
gate name of the qcs C API or "measure" (params = (clbit,)). Every generator
takes a seed and is deterministic (numpy PCG64).
"""

from __future__ import annotations

import math

import numpy as np

from . import GATES

TWO_PI = 2.0 * math.pi


def layered_u3_cz(n: int = 20, depth: int = 20, seed: int = 1, measure: bool = False):
    """20-qubit plain-method workload: each layer applies U3(theta, phi,
    lambda) to every qubit (angles uniform in [0, 2pi)), then CZ on (i, i+1)
    for even i on even layers and odd i on odd layers."""
    rng = np.random.default_rng(seed)
    c = []
    for layer in range(depth):
        ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
        for q in range(n):
            c.append(("u3", tuple(ang[q]), (q,), (), ()))
        for i in range(layer % 2, n - 1, 2):
            c.append(("z", (), (i + 1,), (), (i,)))
    if measure:
        for q in range(n):
            c.append(("measure", (q,), (q,), (), ()))
    return c


def layered_u3_cz_cx_toffoli(n: int = 30, depth: int = 40, seed: int = 1):
    """30-qubit plain-method workload at scale: the U3 layer above; even
    layers add CZ(i, i+1) for even i, odd layers CX(i -> i+1) for odd i; every
    layer ends with one Toffoli on three seeded distinct qubits (two controls,
    one target)."""
    rng = np.random.default_rng(seed)
    c = []
    for layer in range(depth):
        ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
        for q in range(n):
            c.append(("u3", tuple(ang[q]), (q,), (), ()))
        if layer % 2 == 0:
            for i in range(0, n - 1, 2):
                c.append(("z", (), (i + 1,), (), (i,)))
        else:
            for i in range(1, n - 1, 2):
                c.append(("x", (), (i + 1,), (), (i,)))
        a, b, t = (int(v) for v in rng.choice(n, size=3, replace=False))
        c.append(("x", (), (t,), (), (a, b)))
    return c


def u3_random_matching(n: int = 30, layers: int = 60, seed: int = 1):
    """Fusion workload: U3 on every qubit, then CX on a seeded random perfect
    matching of the qubits (n/2 pairs), per layer."""
    rng = np.random.default_rng(seed)
    c = []
    for _ in range(layers):
        ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
        for q in range(n):
            c.append(("u3", tuple(ang[q]), (q,), (), ()))
        perm = rng.permutation(n)
        for k in range(0, n - 1, 2):
            c.append(("x", (), (int(perm[k + 1]),), (), (int(perm[k]),)))
    return c


def qft(n: int, seed: int = 1, swaps: bool = True):
    """Quantum Fourier transform of a seeded random basis state |x>: X on the
    set bits of x, then for j = n-1 .. 0: H(j) and controlled-phase
    2*pi/2^(j-k+1) from every k < j, then the qubit-reversal swaps."""
    rng = np.random.default_rng(seed)
    x = int(rng.integers(0, 1 << min(n, 62)))
    c = []
    for q in range(n):
        if (x >> q) & 1:
            c.append(("x", (), (q,), (), ()))
    for j in range(n - 1, -1, -1):
        c.append(("h", (), (j,), (), ()))
        for k in range(j - 1, -1, -1):
            c.append(("p", (TWO_PI / (1 << (j - k + 1)) if j - k + 1 < 63 else 0.0,), (j,), (), (k,)))
    if swaps:
        for q in range(n // 2):
            c.append(("swap", (), (q, n - 1 - q), (), ()))
    return c, x


def random_circuit(n: int, num_gates: int, seed: int, max_controls: int = 2, gates=None, measure_prob: float = 0.0):
    """Random gates of every kind on random targets, with random positive and
    negative controls; optional interleaved measurements."""
    rng = np.random.default_rng(seed)
    names = list(gates or GATES.keys())
    c = []
    clbit = 0
    for _ in range(num_gates):
        if measure_prob and rng.random() < measure_prob:
            q = int(rng.integers(0, n))
            c.append(("measure", (clbit % n,), (q,), (), ()))
            clbit += 1
            continue
        name = names[int(rng.integers(0, len(names)))]
        npar, nt = GATES[name]
        if nt > n:
            continue
        free = n - nt
        nctl = int(rng.integers(0, min(max_controls, free) + 1))
        qubits = [int(v) for v in rng.choice(n, size=nt + nctl, replace=False)]
        targets = tuple(qubits[:nt])
        ctl_qubits = qubits[nt:]
        neg = tuple(q for q in ctl_qubits if rng.random() < 0.4)
        pos = tuple(q for q in ctl_qubits if q not in neg)
        params = tuple(rng.uniform(-TWO_PI, TWO_PI, size=npar))
        c.append((name, params, targets, neg, pos))
    return c


def hea_circuit(n: int, depth: int, seed: int):
    """Hardware-efficient ansatz: per layer RY(theta) then RZ(phi) on every
    qubit (angles uniform in [-pi, pi]), then a CX ladder 0->1->...->n-1."""
    rng = np.random.default_rng(seed)
    c = []
    for _ in range(depth):
        th = rng.uniform(-math.pi, math.pi, size=n)
        ph = rng.uniform(-math.pi, math.pi, size=n)
        for q in range(n):
            c.append(("ry", (float(th[q]),), (q,), (), ()))
            c.append(("rz", (float(ph[q]),), (q,), (), ()))
        for q in range(n - 1):
            c.append(("x", (), (q + 1,), (), (q,)))
    return c


def to_gatelist(circuit, num_qubits: int, num_clbits: int) -> str:
    """Text form read by examples/gatelist.c (the bin/qcs plug-in)."""
    lines = [f"{num_qubits} {num_clbits}"]
    for op, params, targets, neg, pos in circuit:
        if op == "measure":
            lines.append(f"measure {targets[0]} {int(params[0])}")
            continue
        parts = [op, str(len(params))] + [repr(float(p)) for p in params]
        for group in (targets, neg, pos):
            parts += [str(len(group))] + [str(q) for q in group]
        lines.append(" ".join(parts))
    return "\n".join(lines) + "\n"


def algorithmic_bytes(circuit, n: int, bytes_per_amp: int = 16) -> float:
    """Sum over gates of 2 * bytes_per_amp * (amplitudes the gate can change):
    dense and permuting 1-qubit gates change 2^(n-c) amplitudes, one-sided
    diagonals (z, s, t, p, ...) 2^(n-c-1), swap-like 2-qubit gates
    2^(n-c-1), other 2-qubit gates 2^(n-c); c counts the controls."""
    one_sided = {"z", "s", "sdg", "t", "tdg", "u1", "p"}
    half_two = {"swap", "iswap", "xx_plus_yy", "xx_minus_yy"}
    total = 0.0
    for op, params, targets, neg, pos in circuit:
        if op == "measure" or op == "id":
            continue
        c = len(neg) + len(pos)
        if op == "global_phase":
            amps = 2.0 ** (n - c)
        elif op in one_sided:
            amps = 2.0 ** (n - c - 1)
        elif op in half_two:
            amps = 2.0 ** (n - c - 1)
        elif op == "rccx":
            amps = 3 * 2.0 ** (n - c - 3)
        elif op == "rcccx":
            amps = 4 * 2.0 ** (n - c - 4)
        elif op == "dcx":
            amps = 3 * 2.0 ** (n - c - 2)
        else:
            amps = 2.0 ** (n - c)
        total += 2.0 * bytes_per_amp * amps
    return total
