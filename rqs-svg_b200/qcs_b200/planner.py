"""Self-recorded pass timings and training of the learned cost model.

The simulator times every fused pass it launches while kernel timing is on,
with the pass's features as it ran (block width: 1 on the register path, 3
or 4 for 8 x 8 or 16 x 16 tensor stages; blocks, i.e. stages; arithmetic
gates; light ops -- diagonal phases and permutations; target-qubit stride,
log2 of the largest stride among the pass's local qubits; log2 of the chunk
count n - k, capped at 16, beyond which passes stream and the count no
longer matters). `collect_pass_timings` runs seeded circuits (layered
families and random mixes) with varied pass sizes and execution paths on
registers of several sizes to gather many such samples; `train_cost_model` fits the MLP on log(ns per
amplitude) with the library's own CUDA kernels. A model is trained on one
amplitude type (its dtype).
"""

from __future__ import annotations

import numpy as np

from . import (FUSION_GREEDY, PASS_FEATURES, TENSOR_ALWAYS, TENSOR_ALWAYS_8X8, TENSOR_AUTO, TENSOR_NEVER, CostModel,
               Library, Simulator)
from . import circuits as C

_MIX = ["u3", "x", "h", "rz", "p", "ry", "swap", "rzz", "rxx", "sx"]


def collect_pass_timings(lib: Library, n, min_samples: int, seed: int = 1, max_rounds: int = 100000,
                         precision: int = 128):
    """Return (features [N x PASS_FEATURES] float32, target [N] float32 = log(ns/amp)),
    recorded on registers of n qubits (an int or a list of sizes, which share
    the samples equally)."""
    sizes = [n] if isinstance(n, int) else list(n)
    per = -(-min_samples // len(sizes))
    parts = [_collect(lib, m, per, seed + i, max_rounds, precision) for i, m in enumerate(sizes)]
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])


def _collect(lib: Library, n: int, min_samples: int, seed: int, max_rounds: int, precision: int):
    rng = np.random.default_rng(seed)
    feats, targets = [], []
    total = 0
    with Simulator(lib, n, fusion=FUSION_GREEDY, precision=precision) as sim:
        sim.set_kernel_timing(True)
        rounds = 0
        while total < min_samples and rounds < max_rounds:
            rounds += 1
            max_ops = int(rng.integers(1, 257))
            # the planner's passes keep 11 local qubits; every execution path
            # is recorded: register, 16 x 16 and 8 x 8 tensor stages
            sim.set_planner_options(max_ops, 11)
            sim.set_tensor_passes(int(rng.choice([TENSOR_NEVER, TENSOR_ALWAYS, TENSOR_ALWAYS_8X8])))
            # half the rounds replay layered families (one-qubit layers with
            # CZ / CX / Toffoli or random matchings), the others random mixes
            cseed = int(rng.integers(1 << 30))
            family = int(rng.integers(0, 4))
            if family == 0:
                circ = C.layered_u3_cz_cx_toffoli(n, int(rng.integers(2, 13)), seed=cseed)
            elif family == 1:
                circ = C.u3_random_matching(n, int(rng.integers(2, 13)), seed=cseed)
            else:
                gates = list(rng.choice(_MIX, size=int(rng.integers(2, len(_MIX) + 1)), replace=False))
                circ = C.random_circuit(n, int(rng.integers(64, 400)), seed=cseed,
                                        max_controls=int(rng.integers(0, 3)), gates=gates)
            sim.run(circ)
            sim.synchronize()
            f, ms = sim.pass_records()
            if len(ms):
                feats.append(f)
                targets.append(np.log(ms.astype(np.float64) * 1e6 / float(1 << n)).astype(np.float32))
                total += len(ms)
        sim.set_kernel_timing(False)
        sim.set_planner_options(0, 0)
        sim.set_tensor_passes(TENSOR_AUTO)
    if not feats:
        return np.zeros((0, PASS_FEATURES), np.float32), np.zeros(0, np.float32)
    return np.concatenate(feats), np.concatenate(targets)


def train_cost_model(lib: Library, features, targets, epochs: int = 150, batch: int = 256, lr: float = 2e-3,
                     seed: int = 7):
    model = CostModel(lib, seed)
    loss = model.train(features, targets, epochs=epochs, batch=batch, lr=lr)
    return model, loss


def predicted_pass_ms(model: CostModel, features, n: int) -> np.ndarray:
    return np.exp(model.predict(features).astype(np.float64)) * float(1 << n) * 1e-6


def relative_error(model: CostModel, features, targets) -> float:
    """Median |predicted / measured - 1| of the time per amplitude."""
    pred = model.predict(features).astype(np.float64)
    return float(np.median(np.abs(np.exp(pred - np.asarray(targets, np.float64)) - 1.0)))


__all__ = ["collect_pass_timings", "train_cost_model", "predicted_pass_ms", "relative_error"]
