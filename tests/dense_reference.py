"""Independent numpy statement of the gate unitaries (test helper).

Each matrix is written from the gate's definition (row = output sub-index,
column = input sub-index, bit i of a sub-index = target i), and applied by
brute force over every basis index. Used to check the C++ oracle's
formula-by-formula restatement with a different mechanism.
"""

import cmath
import math

import numpy as np

R2 = 1.0 / math.sqrt(2.0)


def unitary(name, p):
    c = lambda t: math.cos(0.5 * t)  # noqa: E731
    s = lambda t: math.sin(0.5 * t)  # noqa: E731
    e = lambda x: cmath.exp(1j * x)  # noqa: E731
    I2 = np.eye(2, dtype=complex)
    if name == "global_phase":
        return np.array([[e(p[0])]])
    if name in ("u3", "u"):
        th, ph, la = p
        return np.array([[c(th), -e(la) * s(th)], [e(ph) * s(th), e(ph + la) * c(th)]])
    if name == "u4":
        th, ph, la, ga = p
        return e(ga) * np.array([[c(th), -e(la) * s(th)], [e(ph) * s(th), e(ph + la) * c(th)]])
    if name == "u2":
        ph, la = p
        return R2 * np.array([[1, -e(la)], [e(ph), e(ph + la)]])
    if name in ("u1", "p"):
        return np.diag([1, e(p[0])])
    if name == "h":
        return R2 * np.array([[1, 1], [1, -1]])
    if name == "x":
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if name == "y":
        return np.array([[0, -1j], [1j, 0]])
    if name == "z":
        return np.diag([1, -1]).astype(complex)
    if name == "s":
        return np.diag([1, 1j])
    if name == "sdg":
        return np.diag([1, -1j])
    if name == "t":
        return np.diag([1, e(math.pi / 4)])
    if name == "tdg":
        return np.diag([1, e(-math.pi / 4)])
    if name == "sx":
        return 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]])
    if name == "sxdg":
        return 0.5 * np.array([[1 - 1j, 1 + 1j], [1 + 1j, 1 - 1j]])
    if name == "id":
        return I2
    if name == "rx":
        t = p[0]
        return np.array([[c(t), -1j * s(t)], [-1j * s(t), c(t)]])
    if name == "ry":
        t = p[0]
        return np.array([[c(t), -s(t)], [s(t), c(t)]], dtype=complex)
    if name == "rz":
        return np.diag([e(-0.5 * p[0]), e(0.5 * p[0])])
    if name == "r":
        t, ph = p
        return np.array([[c(t), -1j * e(-ph) * s(t)], [-1j * e(ph) * s(t), c(t)]])
    X = np.array([[0, 1], [1, 0]], dtype=complex)
    Y = np.array([[0, -1j], [1j, 0]])
    Z = np.diag([1, -1]).astype(complex)
    # two-target operators: kron(op on target 1, op on target 0)
    k = lambda a1, a0: np.kron(a1, a0)  # noqa: E731
    if name == "swap":
        return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
    if name == "iswap":
        return np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]])
    if name == "rxx":
        t = p[0]
        return c(t) * np.eye(4) - 1j * s(t) * k(X, X)
    if name == "ryy":
        t = p[0]
        return c(t) * np.eye(4) - 1j * s(t) * k(Y, Y)
    if name == "rzz":
        t = p[0]
        return c(t) * np.eye(4) - 1j * s(t) * k(Z, Z)
    if name == "rzx":
        # exp(-i t/2 Z_{target0} X_{target1})
        t = p[0]
        return c(t) * np.eye(4) - 1j * s(t) * k(X, Z)
    if name in ("xx_plus_yy", "xx_minus_yy"):
        t, b = p
        m = np.eye(4, dtype=complex)
        lo, hi = (1, 2) if name == "xx_plus_yy" else (0, 3)
        m[lo, lo] = m[hi, hi] = c(t)
        m[lo, hi] = -1j * s(t) * e(-b)
        m[hi, lo] = -1j * s(t) * e(b)
        return m
    if name == "dcx":
        # CX(target0 -> target1) then CX(target1 -> target0)
        m = np.zeros((4, 4), dtype=complex)
        for sub in range(4):
            b0, b1 = sub & 1, sub >> 1
            b1 ^= b0
            b0 ^= b1
            m[b0 | (b1 << 1), sub] = 1
        return m
    if name == "ecr":
        return R2 * np.array([[0, 1, 0, 1j], [1, 0, -1j, 0], [0, 1j, 0, 1], [-1j, 0, 1, 0]])
    if name == "rccx":
        m = np.eye(8, dtype=complex)
        m[3, 3] = 0
        m[7, 7] = 0
        m[3, 7] = -1j
        m[7, 3] = 1j
        m[5, 5] = -1
        return m
    if name == "rcccx":
        m = np.eye(16, dtype=complex)
        m[3, 3] = 1j
        m[7, 7] = 0
        m[15, 15] = 0
        m[7, 15] = 1
        m[15, 7] = -1
        m[11, 11] = -1j
        return m
    raise KeyError(name)


def apply(state, n, name, params, targets, negctrls=(), ctrls=()):
    """Brute-force application on a logical-order state vector."""
    u = unitary(name, params)
    d = 1 << len(targets)
    out = state.copy()
    tmask = 0
    for t in targets:
        tmask |= 1 << t
    for base in range(1 << n):
        if base & tmask:
            continue
        if any((base >> q) & 1 for q in negctrls) or not all((base >> q) & 1 for q in ctrls):
            continue
        idx = []
        for sub in range(d):
            i = base
            for b, t in enumerate(targets):
                if (sub >> b) & 1:
                    i |= 1 << t
            idx.append(i)
        v = state[idx]
        out[idx] = u @ v
    return out
