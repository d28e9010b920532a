"""Learned cost model and planner on the GPU.

- the CUDA backward pass equals the float64 numpy restatement
  (oracle/mlp_oracle.py) on the same parameters and batch;
- training with the CUDA kernels drives the loss down on recorded timings;
- the learned planner changes only how gates are cut into passes: its
  results equal the oracle's, on the learned plan and on the greedy plan
  the judge runs next for comparison.
"""

import sys
from pathlib import Path

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import FUSION_LEARNED
from qcs_b200 import circuits as C
from qcs_b200 import planner

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def test_cost_model_gradients_match_numpy(gpu_lib):
    model = qcs_b200.CostModel(gpu_lib, seed=3)
    try:
        params, _ = model.params()
        rng = np.random.default_rng(0)
        for B in (1, 17, 256):
            x = rng.normal(size=(B, qcs_b200.PASS_FEATURES)).astype(np.float32)
            t = rng.normal(size=B).astype(np.float32)
            g, loss = model.gradients(x, t)
            ref_loss, ref_g = mlp_oracle.loss_and_gradients(params, x, t)
            assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
            scale = max(1e-6, float(np.max(np.abs(ref_g))))
            assert np.max(np.abs(g - ref_g)) <= 1e-4 * scale, B
    finally:
        model.close()


def test_cost_model_learns_a_smooth_function(gpu_lib):
    rng = np.random.default_rng(1)
    x = rng.uniform([1, 1, 3, 1, 10, 16], [4, 8, 30, 64, 29, 16], size=(4096, 6)).astype(np.float32)
    t = (0.05 * x[:, 3] + 0.3 * np.sin(x[:, 2] / 5.0) - 0.1 * (x[:, 0] - 2) + 0.02 * x[:, 1]).astype(np.float32)
    model = qcs_b200.CostModel(gpu_lib, seed=2)
    try:
        loss = model.train(x, t, epochs=60, batch=128, lr=3e-3)
        assert loss < 0.01   # standardised MSE
        pred = model.predict(x)
        assert np.sqrt(np.mean((pred - t) ** 2)) < 0.05 * float(np.std(t)) * 3
    finally:
        model.close()


def test_pass_timings_and_learned_plans_keep_results_exact(gpu_lib, oracle_lib):
    n = 18
    feats, target = planner.collect_pass_timings(gpu_lib, n, min_samples=1500, seed=4)
    assert len(target) >= 1500
    # every execution path was recorded: register (1), 8 x 8 (3), 16 x 16 (4)
    assert set(np.unique(feats[:, 0]).tolist()) == {1.0, 3.0, 4.0}
    assert np.all(feats[:, 1] >= 1)                 # stages
    assert np.all(feats[:, 4] <= n - 1)             # highest local qubit
    assert np.all(feats[:, 5] == n - 11)            # log2 of the chunk count
    model, loss = planner.train_cost_model(gpu_lib, feats, target, epochs=40)
    try:
        assert loss < 1.0
        circ = C.qft(n, seed=5)[0] + C.layered_u3_cz_cx_toffoli(n, 4, seed=6)
        with qcs_b200.Simulator(oracle_lib, n) as sim:
            sim.run(circ)
            ref = sim.statevector()
        with qcs_b200.Simulator(gpu_lib, n, fusion=FUSION_LEARNED) as sim:
            sim.set_cost_model(model)
            plans = []
            for _ in range(3):
                sim.set_state("zero")
                sim.run(circ)
                got = sim.statevector()
                plans.append(sim.planner_judge())
                assert np.max(np.abs(got - ref)) <= 1e-12
            # first flush: learned plan; second: greedy for comparison; third:
            # the faster of the two measured times
            assert plans[0]["learned_plan"] and not plans[1]["learned_plan"]
            assert plans[2]["greedy_ms"] > 0 and plans[2]["learned_ms"] > 0
            faster_learned = plans[2]["learned_ms"] <= plans[2]["greedy_ms"]
            assert plans[2]["learned_plan"] == faster_learned
    finally:
        model.close()
