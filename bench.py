"""Benchmark: 30-qubit plain-method circuit at scale (complex128).

Workload (one step): the 30-qubit layered circuit of depth 40 -- U3 on every
qubit per layer, CZ(i, i+1) for even i on even layers, CX(i -> i+1) for odd i
on odd layers, one seeded Toffoli per layer (1820 gates) -- applied to
|0...0>, followed by <Z_q> for all 30 qubits and 4096 shots drawn with the
measurement chain rule. The state is 2^30 complex128 = 16 GiB, far larger
than L2, so no flush is needed between steps.

metric: circuit wall seconds per step (device time between CUDA events on the
library's stream), lower is better; with N GPUs each rank runs its own
replica ("replicas only": the path has no exchange step) and value is the
slowest rank's time divided by N (seconds per circuit for the whole job).

Arms:
  default             this library (fused greedy passes; --fusion plain for the
                      one-kernel-per-gate path)
  --impl reference    the reference library built from its sources for
                      sm_100a (oracle/_ref/libqcs_ref.so) on the same GPU, same
                      circuit, through its C API; it has no <Z> or sampler, so
                      its step is the circuit plus one measurement of every
                      qubit (one bin/qcs sample). Without that build the CPU
                      oracle runs a bounded sample instead.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "rqs-svg_b200"))

WORLD = int(os.environ.get("WORLD_SIZE", "1"))
RANK = int(os.environ.get("RANK", "0"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
if WORLD > 1:
    # one GPU per process: the library uses the current (first visible) device
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = vis.split(",") if vis else [str(i) for i in range(64)]
    os.environ["CUDA_VISIBLE_DEVICES"] = devs[LOCAL_RANK]

import numpy as np  # noqa: E402

import qcs_b200  # noqa: E402
from qcs_b200 import circuits as C  # noqa: E402

PEAKS = REPO / "MEASURED_PEAKS.json"
TRAFFIC_FILE = REPO / "profiles" / "fused_pass_traffic.txt"
FALLBACK_HBM = 6650.0
SHOTS = 4096


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--fusion", choices=["plain", "greedy"], default="greedy")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--no-plain-compare", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-peak", action="store_true")
    return ap.parse_args()


def hbm_peak():
    try:
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def traffic_per_launch(n):
    """dram read+write bytes of one fused pass from the committed ncu summary
    (scaled by 2^n from the captured size)."""
    try:
        for line in TRAFFIC_FILE.read_text().splitlines():
            if line.startswith("traffic_bytes_per_amplitude:"):
                return float(line.split(":")[1]) * (1 << n)
    except Exception:
        pass
    return None


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, device_index):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append(parts)
        os.unlink(self.file.name)
        mine = [r for r in rows if r[0] == str(device_index)] or rows
        if not mine:
            return None
        sm = [float(r[1]) for r in mine if r[1].replace(".", "").isdigit()]
        maxsm = [float(r[2]) for r in mine if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in mine for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if maxsm and s > 0.5 * max(maxsm)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(maxsm) if maxsm else None, "reasons": reasons, "samples": len(mine)}


def dist_init(backend="nccl"):
    """One process per GPU (replicas): the group only carries the barrier
    and the max-over-ranks of the timings. nccl on GPUs, gloo on CPU."""
    if WORLD == 1:
        return None
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    if backend == "nccl":
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", 0))
    else:
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return dist


def _device(dist):
    return "cuda" if dist is not None and dist.get_backend() == "nccl" else "cpu"


def barrier(dist):
    if dist is not None:
        import torch

        dist.barrier()
        if _device(dist) == "cuda":
            torch.cuda.synchronize()


def max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_replica_times(dist, per_step_seconds, world):
    """Whole-job numbers from each rank's per-step device times: the slowest
    rank's total, seconds per step, and seconds per circuit for the job
    (world replicas ran one circuit per step each)."""
    total = max_over_ranks(dist, float(sum(per_step_seconds)))
    steps = len(per_step_seconds)
    return {"total_s": total, "sec_per_step": total / steps, "value": total / steps / world}


def run_step(sim, circuit, with_outputs=True):
    sim.set_state("zero")
    sim.run(circuit)
    if with_outputs:
        z, norm = sim.expectation_z()
        shots = sim.sample(SHOTS)
        return z, norm, shots
    sim.synchronize()
    return None


def fp64_flops(circuit, n):
    """Useful FP64 flops of one step: a dense 2x2 complex gate costs 16
    flops per amplitude of its control subspace (four complex multiply-adds
    per pair), a one-sided phase 6 per changed amplitude; permutations (X,
    CX, Toffoli, SWAP) cost none."""
    one_sided = {"z", "s", "sdg", "t", "tdg", "u1", "p"}
    perm = {"x", "swap", "id"}
    total = 0.0
    for op, params, targets, neg, pos in circuit:
        c = len(neg) + len(pos)
        if op in perm or op == "measure":
            continue
        if op in one_sided:
            total += 6.0 * 2.0 ** (n - c - 1)
        else:
            total += 16.0 * 2.0 ** (n - c)
    return total


def dgemm_peak_tflops():
    """FP64 peak of this GPU, measured as cuBLAS DGEMM (8192^3) throughput."""
    try:
        import torch

        a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = None
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            torch.cuda.synchronize()
            t = s.elapsed_time(e) * 1e-3
            best = t if best is None else min(best, t)
        del a, b
        torch.cuda.empty_cache()
        return 2 * 8192 ** 3 / best / 1e12
    except Exception:
        return None


def cpu_baseline(n_full, depth):
    """The CPU oracle (OpenMP over all host cores) on a bounded sample: the
    first two layers of the same circuit at 28 qubits, scaled to the full
    30-qubit circuit by algorithmic bytes."""
    oracle_so = REPO / "oracle" / "liboracle_qcs.so"
    if not oracle_so.exists():
        return None
    n = min(28, n_full)
    lib = qcs_b200.Library(oracle_so)
    full = C.layered_u3_cz_cx_toffoli(n_full, depth, seed=1)
    sample = C.layered_u3_cz_cx_toffoli(n, 2, seed=1)
    with qcs_b200.Simulator(lib, n) as sim:
        t0 = time.perf_counter()
        sim.run(sample)
        dt = time.perf_counter() - t0
    bytes_sample = C.algorithmic_bytes(sample, n)
    bytes_full = C.algorithmic_bytes(full, n_full)
    return {"value": dt * bytes_full / bytes_sample, "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first 2 layers ({len(sample)} gates) of the circuit at {n} qubits on the CPU oracle, "
                      f"{dt:.1f} s, scaled to the 30-qubit circuit by algorithmic bytes"}


def main():
    args = parse_args()
    dist = dist_init()
    n, depth = args.qubits, args.depth
    circuit = C.layered_u3_cz_cx_toffoli(n, depth, seed=1)
    alg_bytes = C.algorithmic_bytes(circuit, n)
    workload = (f"layered U3 + CZ/CX + Toffoli, {n} qubits, depth {depth}, complex128, "
                f"|0..0> -> <Z_q> x{n} + {SHOTS} shots")
    if args.impl == "reference":
        return run_reference(args, dist, circuit, workload)

    lib = qcs_b200.Library(qcs_b200.LIB_PATH)
    fusion = qcs_b200.FUSION_GREEDY if args.fusion == "greedy" else qcs_b200.FUSION_PLAIN
    sim = qcs_b200.Simulator(lib, n, seed=1234 + RANK, fusion=fusion)
    for _ in range(args.warmup):
        run_step(sim, circuit)
    e0, e1 = sim.event_create(), sim.event_create()
    clocks = Clocks()
    barrier(dist)
    clocks.start()
    sim.set_kernel_timing(True)
    sim.reset_stats()
    per_step = []
    for _ in range(args.steps):
        sim.event_record(e0)
        run_step(sim, circuit)
        sim.event_record(e1)
        per_step.append(sim.elapsed(e0, e1))
    barrier(dist)
    ktimes = sim.kernel_times()
    pass_feats, pass_ms = sim.pass_records()
    sim.set_kernel_timing(False)
    stats = sim.stats()
    clk = clocks.stop(0)
    agg = aggregate_replica_times(dist, per_step, WORLD)
    sec_per_step = agg["sec_per_step"]
    passes = None
    if len(pass_ms):
        passes = {"per_step": len(pass_ms) / args.steps, "median_ms": float(np.median(pass_ms)),
                  "max_ms": float(np.max(pass_ms)), "gates_per_pass": float(np.mean(pass_feats[:, 2])),
                  "hbm_floor_ms": 2 * 16 * (1 << n) / (hbm_peak()[0] * 1e9) * 1e3}

    # end to end through the C ABI: host wall clock, host inputs (gate
    # parameters, sampler uniforms) in, results (<Z>, shots) out
    barrier(dist)
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run_step(sim, circuit)
        e2e.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(dist, sum(e2e))
    nparams = sum(len(p) for _, p, *_ in circuit)
    h2d = SHOTS * n * 8 + nparams * 8
    d2h = (n + 1) * 8 + SHOTS * 8

    plain = None
    if fusion == qcs_b200.FUSION_GREEDY and not args.no_plain_compare and WORLD == 1:
        sim.set_fusion(qcs_b200.FUSION_PLAIN)
        run_step(sim, circuit, with_outputs=False)
        sim.set_kernel_timing(True)
        sim.event_record(e0)
        run_step(sim, circuit)
        sim.event_record(e1)
        t_plain = sim.elapsed(e0, e1)
        kt = sim.kernel_times()
        sim.set_kernel_timing(False)
        peak, _ = hbm_peak()
        gbs = kt["plain_bytes"] / (kt["plain_ms"] * 1e-3) / 1e9 if kt["plain_ms"] else None
        plain = {"value": t_plain, "unit": "s", "gate_kernels": kt["plain_launches"],
                 "hbm_gbs": gbs, "frac_of_measured_hbm": gbs / peak if gbs else None,
                 "frac_of_8tbs": gbs / 8000.0 if gbs else None,
                 "speedup_fused_vs_plain": t_plain / sec_per_step}
        sim.set_fusion(fusion)
    sim.close()

    peak, peak_kind = hbm_peak()
    if fusion == qcs_b200.FUSION_GREEDY and ktimes["fused_launches"]:
        launches, ms, by = ktimes["fused_launches"], ktimes["fused_ms"], ktimes["fused_bytes"]
        kernel = "fused_pass_kernel"
    else:
        launches, ms, by = ktimes["plain_launches"], ktimes["plain_ms"], ktimes["plain_bytes"]
        kernel = "gate_plain_kernel"
    achieved = (by / launches) / (ms / launches * 1e-3) / 1e9 if launches else 0.0
    traffic = traffic_per_launch(n) if kernel == "fused_pass_kernel" else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} (copy, MEASURED_PEAKS hbm_gbs)" if peak_kind == "measured" else "fallback",
                "frac_of_8tbs": achieved / 8000.0, "traffic": traffic,
                "launches": launches, "avg_launch_ms": ms / launches if launches else None,
                "algorithmic_bytes_per_launch": by / launches if launches else None}
    cpu = None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(n, depth)
    fp64 = None
    if RANK == 0 and WORLD == 1 and not args.no_fp64_peak:
        flops = fp64_flops(circuit, n)
        peak_tf = dgemm_peak_tflops()
        fp64 = {"achieved_tflops": flops / sec_per_step / 1e12, "useful_flops_per_step": flops,
                "peak_tflops": peak_tf, "peak_kind": "measured: cuBLAS DGEMM 8192^3 (torch.matmul float64)",
                "frac": (flops / sec_per_step / 1e12) / peak_tf if peak_tf else None}

    line = {
        "metric": f"circuit wall s at {n}q (plain-method circuit at scale)",
        "value": agg["value"],
        "unit": "s",
        "n_gpus": WORLD,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": sec_per_step * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128 (f64)",
        "data": "synthetic (seeded circuit)",
        "config": {"workload": workload, "qubits": n, "depth": depth, "gates": len(circuit), "shots": SHOTS,
                   "fusion": args.fusion, "parallelism": f"replicas x{WORLD}",
                   "l2": "state (16 GiB) larger than L2; no flush"},
        "hbm_gbs_algorithmic": alg_bytes / sec_per_step / 1e9,
        "e2e": {"value": e2e_total / args.steps / WORLD, "unit": "s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(stats["kernel_launches"] / args.steps),
        "roofline": roofline,
        "fp64": fp64,
        "passes": passes,
        "step_s": per_step,
        "cpu_baseline": cpu,
        "plain": plain,
        "clocks": clk,
    }
    if RANK == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_reference(args, dist, circuit, workload):
    n = args.qubits
    ref_so = REPO / "oracle" / "_ref" / "libqcs_ref.so"
    if RANK != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    if ref_so.exists():
        lib = qcs_b200.Library(ref_so)
        sim = qcs_b200.Simulator(lib, n, n)
        meas = [("measure", (q,), (q,), (), ()) for q in range(n)]

        def step():
            sim.reinitialize_mapping()
            sim.set_state("zero")
            sim.reset_clbits()
            sim.reset_measurement_state()
            sim.run(circuit + meas)

        for _ in range(args.warmup):
            step()
        e0, e1 = sim.event_create(), sim.event_create()
        clocks = Clocks()
        clocks.start()
        dev, wall = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            sim.event_record(e0)
            step()
            sim.event_record(e1)
            dev.append(sim.elapsed(e0, e1))
            wall.append(time.perf_counter() - t0)
        clk = clocks.stop(0)
        sim.close()
        value = sum(dev) / args.steps
        line = {"impl": "reference", "metric": f"circuit wall s at {n}q (plain-method circuit at scale)",
                "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "c128 (f64)", "data": "synthetic (seeded circuit)",
                "config": {"workload": workload.replace(f"<Z_q> x{n} + {SHOTS} shots", "one measurement of every qubit"),
                           "qubits": n, "depth": args.depth, "gates": len(circuit)},
                "e2e": {"value": sum(wall) / args.steps, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                                 "sample": "reference library built from its sources for sm_100a, run on the GPU "
                                           "(it has no CPU path); host thread count 1"},
                "clocks": clk}
    else:
        cpu = cpu_baseline(n, args.depth)
        line = {"impl": "reference", "metric": f"circuit wall s at {n}q (plain-method circuit at scale)",
                "value": cpu["value"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)",
                "data": "synthetic (seeded circuit)", "config": {"workload": workload},
                "e2e": {"value": cpu["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
