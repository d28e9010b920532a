"""Benchmark: 30-qubit plain-method circuit at scale (complex128).

Workload (one step, default --workload layered): the 30-qubit layered circuit
of depth 40 -- U3 on every qubit per layer, CZ(i, i+1) for even i on even
layers, CX(i -> i+1) for odd i on odd layers, one seeded Toffoli per layer
(1820 gates) -- applied to |0...0>, followed by <Z_q> for all 30 qubits and
4096 shots drawn with the measurement chain rule. The state is 2^30
complex128 = 16 GiB, far larger than L2, so no flush is needed between steps.

Other workloads (same line format; they check accuracy against the
complex128 plain path, or against the closed form for the QFT):
  --workload matching   U3 + CX on seeded random perfect matchings, 60 layers
                        (--precision 64 for complex64 registers)
  --workload qft        QFT of a seeded random basis state (33 qubits with
                        --qubits 33); --fusion learned first records pass
                        timings on a --train-qubits register, trains the cost
                        model on the GPU and lets its planner compete with the
                        greedy one

metric: circuit wall seconds per step (device time between CUDA events on the
library's stream), lower is better; with N GPUs each rank runs its own
replica ("replicas only": the path has no exchange step) and value is the
slowest rank's time divided by N (seconds per circuit for the whole job).

Arms:
  default             this library (fused passes under the learned planner and
                      its judge; --fusion greedy for the greedy planner alone,
                      --fusion plain for the one-kernel-per-gate path)
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
FALLBACK_HBM = 6650.0
SHOTS = 4096


def _layered(n, depth):
    return C.layered_u3_cz_cx_toffoli(n, depth, seed=1)


def _matching(n, depth):
    return C.u3_random_matching(n, depth, seed=1)


def _qft(n, depth):
    return C.qft(n, seed=1)[0]


# name: (generator(n, depth), default depth, description, draws shots)
BATCH_CIRCUITS = 4096
CLI_SAMPLES = 1024
WORKLOADS = {
    "cli": (None, 20, "bin/qcs -s " + str(CLI_SAMPLES) + " on a circuit plug-in: layered U3 + CZ, {n} qubits, "
                      "depth {d}, {p}, then a measurement of every qubit; each sample re-runs the circuit",
            False),
    "hea_batch": (None, 8, "{c} hardware-efficient-ansatz circuits (RY, RZ on every qubit, "
                           "CX ladder per layer), widths uniform in 10..20, depth {d}, {p}, new parameters "
                           "every step -> <Z_q> of every circuit", False),
    "layered": (_layered, 40, "layered U3 + CZ/CX + Toffoli, {n} qubits, depth {d}, {p}, "
                              "|0..0> -> <Z_q> x{n} + " + str(SHOTS) + " shots", True),
    "matching": (_matching, 60, "U3 on every qubit + CX on a seeded random perfect matching, {n} qubits, "
                                "{d} layers, {p}, |0..0> -> <Z_q> x{n}", False),
    "qft": (_qft, 0, "QFT of a seeded random basis state (X on its set bits, H + controlled phases, "
                     "qubit-reversal swaps), {n} qubits, {p} -> <Z_q> x{n}", False),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="layered",
                    help="layered: U3 + CZ/CX + Toffoli layers with <Z> and shots (default); "
                         "matching: U3 + CX on random matchings; qft: QFT of a random basis state")
    ap.add_argument("--fusion", choices=["plain", "greedy", "learned"], default="learned",
                    help="learned (default): the cost model is trained on pass timings recorded on smaller "
                         "registers, its plan and the greedy plan are both timed during warm-up and the faster "
                         "one runs; greedy: fused passes cut greedily; plain: one kernel per gate")
    ap.add_argument("--tensor", choices=["never", "auto", "always", "8x8"], default="auto",
                    help="tensor passes (stages as dense matrices on the tensor cores): auto (default) where the "
                         "cost estimate favours them, 16x16 or 8x8 stages; always: 16x16 stages wherever allowed; "
                         "8x8: 8x8 stages wherever allowed")
    ap.add_argument("--batch-tensor", type=int, choices=[0, 1, 2], default=1,
                    help="hea_batch: 0 register passes only, 1 tuned per group (default), 2 tensor passes where allowed")
    ap.add_argument("--engine", choices=["tcgen05", "mma.sync"], default="tcgen05",
                    help="tensor engine of complex64 16x16 stages: tcgen05 (default, where a pass allows it) or "
                         "warp-level mma.sync")
    ap.add_argument("--precision", type=int, choices=[128, 64], default=None,
                    help="amplitude bits (default 128; 64 for hea_batch)")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=None, help="layers (default 40 layered, 60 matching)")
    ap.add_argument("--train-qubits", default="20,22,24,26",
                    help="register sizes (comma-separated) the cost model's timings come from")
    ap.add_argument("--train-samples", type=int, default=20000, help="pass timings recorded to train the cost model")
    ap.add_argument("--batch-circuits", type=int, default=BATCH_CIRCUITS, help="circuits of the hea_batch workload")
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


def traffic_per_launch(n, kernel="fused_pass_kernel"):
    """dram read+write bytes of one pass of this kernel from the committed ncu
    summary profiles/<kernel>_traffic.txt (complex128 bytes per amplitude,
    scaled by 2^n from the captured size), or None."""
    path = REPO / "profiles" / f"{kernel}_traffic.txt"
    try:
        for line in path.read_text().splitlines():
            if line.startswith("traffic_bytes_per_amplitude:"):
                return float(line.split(":")[1]) * (1 << n)
    except Exception:
        pass
    return None


def batch_traffic_per_amplitude():
    """dram read+write bytes per amplitude and pass of the batched 8x8 tensor
    pass (complex64), from profiles/tensor3_pass_kernel_batch_traffic.txt, or None."""
    try:
        for line in (REPO / "profiles" / "tensor3_pass_kernel_batch_traffic.txt").read_text().splitlines():
            if line.startswith("traffic_bytes_per_amplitude_pass:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


def dominant_pass_kernel(stats):
    """The kernel that runs most fused passes: the register pass, or the
    tensor pass of 8x8 stages, of 16x16 stages on mma.sync, or on tcgen05."""
    fused, tensor = stats["fused_passes"], stats["tensor_passes"]
    if tensor * 2 < fused:
        return "fused_pass_kernel"
    t8, tc = stats["tensor8_passes"], stats["tcgen05_passes"]
    t16 = tensor - t8 - tc
    return max([(t8, "tensor3_pass_kernel"), (tc, "tc_pass_kernel"), (t16, "tensor_pass_kernel")])[1]


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


def run_step(sim, circuit, with_outputs=True, shots=True):
    sim.set_state("zero")
    sim.run(circuit)
    if with_outputs:
        z, norm = sim.expectation_z()
        samples = sim.sample(SHOTS) if shots else None
        return z, norm, samples
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


def cpu_baseline(gen, n_full, depth, bytes_per_amp=16):
    """The CPU oracle (OpenMP over all host cores) on a bounded sample: the
    first layers (at most 100 gates) of the same workload at 28 qubits,
    scaled to the full circuit by algorithmic bytes."""
    oracle_so = REPO / "oracle" / "liboracle_qcs.so"
    if not oracle_so.exists():
        return None
    n = min(28, n_full)
    lib = qcs_b200.Library(oracle_so)
    full = gen(n_full, depth)
    sample = gen(n, min(depth, 2))[:100]
    with qcs_b200.Simulator(lib, n) as sim:
        t0 = time.perf_counter()
        sim.run(sample)
        dt = time.perf_counter() - t0
    bytes_sample = C.algorithmic_bytes(sample, n)
    bytes_full = C.algorithmic_bytes(full, n_full)
    return {"value": dt * bytes_full / bytes_sample, "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first {len(sample)} gates of the workload at {n} qubits on the CPU oracle (complex128), "
                      f"{dt:.1f} s, scaled to the {n_full}-qubit circuit by algorithmic bytes"}


def train_planner(lib, args):
    """Record pass timings on a smaller register of the same precision,
    train the cost model with the library's CUDA kernels, and report it."""
    from qcs_b200 import planner

    t0 = time.perf_counter()
    sizes = [int(v) for v in str(args.train_qubits).split(",")]
    feats, target = planner.collect_pass_timings(lib, sizes, args.train_samples, seed=11,
                                                 precision=args.precision)
    t1 = time.perf_counter()
    model, loss = planner.train_cost_model(lib, feats, target, epochs=60)
    t2 = time.perf_counter()
    info = {"timings": int(len(target)), "train_qubits": args.train_qubits, "record_s": t1 - t0,
            "train_s": t2 - t1, "loss": loss, "median_rel_err": planner.relative_error(model, feats, target)}
    return model, info


def qft_spot_check(sim, n, count=4096):
    """Max |a_y - 2^(-n/2) exp(2 pi i x y / 2^n)| over seeded random logical
    indices y, relative to the amplitude modulus 2^(-n/2)."""
    _, x = C.qft(n, seed=1)
    y = np.random.default_rng(99).integers(0, 1 << n, size=count, dtype=np.uint64)
    got = sim.amplitudes(y)
    mask = (1 << n) - 1
    phase = np.array([((x * int(v)) & mask) for v in y], dtype=np.float64) / float(1 << n)
    want = np.exp(2j * np.pi * phase) / math.sqrt(float(1 << n))
    return float(np.max(np.abs(got - want)) * math.sqrt(float(1 << n)))


def main():
    args = parse_args()
    dist = dist_init()
    if args.workload == "hea_batch":
        return main_batch(args, dist)
    if args.workload == "cli":
        return main_cli(args, dist)
    if args.precision is None:
        args.precision = 128
    n = args.qubits
    gen, default_depth, desc, draws_shots = WORKLOADS[args.workload]
    depth = args.depth if args.depth is not None else default_depth
    circuit = gen(n, depth)
    bpa = args.precision // 8
    prec = "complex128" if args.precision == 128 else "complex64"
    alg_bytes = C.algorithmic_bytes(circuit, n, bpa)
    workload = desc.format(n=n, d=depth, p=prec)
    if args.impl == "reference":
        return run_reference(args, dist, circuit, workload, gen, depth)

    lib = qcs_b200.Library(qcs_b200.LIB_PATH)
    fusion = {"plain": qcs_b200.FUSION_PLAIN, "greedy": qcs_b200.FUSION_GREEDY,
              "learned": qcs_b200.FUSION_LEARNED}[args.fusion]
    sim = qcs_b200.Simulator(lib, n, seed=1234 + RANK, fusion=fusion, precision=args.precision)
    sim.set_tensor_passes({"never": qcs_b200.TENSOR_NEVER, "auto": qcs_b200.TENSOR_AUTO,
                           "always": qcs_b200.TENSOR_ALWAYS, "8x8": qcs_b200.TENSOR_ALWAYS_8X8}[args.tensor])
    sim.set_tensor_engine(qcs_b200.ENGINE_TCGEN05 if args.engine == "tcgen05" else qcs_b200.ENGINE_MMA_SYNC)
    model, training, judge = None, None, None
    if fusion == qcs_b200.FUSION_LEARNED:
        model, training = train_planner(lib, args)
        sim.set_cost_model(model)
    # the clock sampler starts before the warm-up, so that its own start-up
    # (nvidia-smi initialising NVML) does not fall into the timed steps; its
    # samples span warm-up and timed steps, all under the same load
    clocks = Clocks()
    clocks.start()
    for _ in range(args.warmup):
        run_step(sim, circuit, shots=draws_shots)
    if fusion == qcs_b200.FUSION_LEARNED:
        # the judge has timed the learned plan and then the greedy plan of
        # this gate queue during warm-up; timed steps run the faster one
        judge = sim.planner_judge()
    e0, e1 = sim.event_create(), sim.event_create()
    barrier(dist)
    sim.set_kernel_timing(True)
    sim.reset_stats()
    per_step = []
    for _ in range(args.steps):
        sim.event_record(e0)
        run_step(sim, circuit, shots=draws_shots)
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
        passes = {"per_step": len(pass_ms) / args.steps, "tensor_per_step": stats["tensor_passes"] / args.steps,
                  "tensor8_per_step": stats["tensor8_passes"] / args.steps,
                  "tcgen05_per_step": stats["tcgen05_passes"] / args.steps,
                  "median_ms": float(np.median(pass_ms)),
                  "max_ms": float(np.max(pass_ms)), "stages_per_pass": float(np.mean(pass_feats[:, 1])),
                  "gates_per_pass": float(np.mean(pass_feats[:, 2])),
                  "light_ops_per_pass": float(np.mean(pass_feats[:, 3])),
                  "hbm_floor_ms": 2 * bpa * (1 << n) / (hbm_peak()[0] * 1e9) * 1e3}

    # end to end through the C ABI: host wall clock, host inputs (gate
    # parameters, sampler uniforms) in, results (<Z>, shots) out
    barrier(dist)
    run_step(sim, circuit, shots=draws_shots)   # untimed warm-up of the host path
    sim.synchronize()
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run_step(sim, circuit, shots=draws_shots)
        e2e.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(dist, sum(e2e))
    nparams = sum(len(p) for _, p, *_ in circuit)
    h2d = (SHOTS * n * 8 if draws_shots else 0) + nparams * 8
    d2h = (n + 1) * 8 + (SHOTS * 8 if draws_shots else 0)

    accuracy, plain = None, None
    if fusion != qcs_b200.FUSION_PLAIN and not args.no_plain_compare and WORLD == 1:
        if args.workload == "qft":
            # a second 2^n register may not fit: check the fused result
            # against the closed form, then time the plain path in place
            accuracy = {"check": "4096 seeded amplitudes vs 2^(-n/2) exp(2 pi i x y / 2^n)",
                        "max_rel_err": qft_spot_check(sim, n)}
            ref = sim
            ref.set_fusion(qcs_b200.FUSION_PLAIN)
        else:
            ref = qcs_b200.Simulator(lib, n, seed=1234, fusion=qcs_b200.FUSION_PLAIN)
        run_step(ref, circuit, with_outputs=False)
        ref.set_kernel_timing(True)
        r0, r1 = ref.event_create(), ref.event_create()
        ref.event_record(r0)
        run_step(ref, circuit, shots=draws_shots)
        ref.event_record(r1)
        t_plain = ref.elapsed(r0, r1)
        kt = ref.kernel_times()
        ref.set_kernel_timing(False)
        if ref is not sim:
            # fused result (this precision) against the complex128 plain path
            run_step(sim, circuit, with_outputs=False)
            cmp = sim.compare(ref)
            accuracy = {"check": "full register vs the complex128 plain path",
                        "fidelity": cmp["fidelity"], "infidelity": 1.0 - cmp["fidelity"],
                        "max_abs_diff": cmp["max_abs_diff"], "norm": cmp["norm_self"],
                        "norm_plain": cmp["norm_other"], "overlap_sq": abs(cmp["overlap"]) ** 2}
            ref.close()
        else:
            sim.set_fusion(fusion)
        peak, _ = hbm_peak()
        gbs = kt["plain_bytes"] / (kt["plain_ms"] * 1e-3) / 1e9 if kt["plain_ms"] else None
        plain = {"value": t_plain, "unit": "s", "precision": "complex128", "gate_kernels": kt["plain_launches"],
                 "hbm_gbs": gbs, "frac_of_measured_hbm": gbs / peak if gbs else None,
                 "frac_of_8tbs": gbs / 8000.0 if gbs else None,
                 "speedup_fused_vs_plain": t_plain / sec_per_step}
    sim.close()
    if model is not None:
        model.close()

    peak, peak_kind = hbm_peak()
    if fusion != qcs_b200.FUSION_PLAIN and ktimes["fused_launches"]:
        # every fused pass (register or tensor) reads and writes the register
        # once; the timings cover all of them, the name says which kernel runs
        # most of them
        launches, ms, by = ktimes["fused_launches"], ktimes["fused_ms"], ktimes["fused_bytes"]
        kernel = dominant_pass_kernel(stats)
    else:
        launches, ms, by = ktimes["plain_launches"], ktimes["plain_ms"], ktimes["plain_bytes"]
        kernel = "gate_plain_kernel"
    achieved = (by / launches) / (ms / launches * 1e-3) / 1e9 if launches else 0.0
    tpl = traffic_per_launch(n, kernel) if kernel != "gate_plain_kernel" else None
    traffic = tpl * bpa / 16 if tpl else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} (copy, MEASURED_PEAKS hbm_gbs)" if peak_kind == "measured" else "fallback",
                "frac_of_8tbs": achieved / 8000.0, "traffic": traffic,
                "launches": launches, "avg_launch_ms": ms / launches if launches else None,
                "algorithmic_bytes_per_launch": by / launches if launches else None}
    cpu = None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(gen, n, depth)
    fp64 = None
    if RANK == 0 and WORLD == 1 and not args.no_fp64_peak and args.precision == 128:
        flops = fp64_flops(circuit, n)
        peak_tf = dgemm_peak_tflops()
        fp64 = {"achieved_tflops": flops / sec_per_step / 1e12, "useful_flops_per_step": flops,
                "peak_tflops": peak_tf, "peak_kind": "measured: cuBLAS DGEMM 8192^3 (torch.matmul float64)",
                "frac": (flops / sec_per_step / 1e12) / peak_tf if peak_tf else None}

    line = {
        "metric": f"circuit wall s at {n}q ({args.workload} workload)",
        "value": agg["value"],
        "unit": "s",
        "n_gpus": WORLD,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": sec_per_step * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128 (f64)" if args.precision == 128 else "c64 (f32 gates, f64 reductions)",
        "data": "synthetic (seeded circuit)",
        "config": {"workload": workload, "qubits": n, "depth": depth, "gates": len(circuit),
                   "shots": SHOTS if draws_shots else 0, "fusion": args.fusion, "tensor_passes": args.tensor,
                   "tensor_engine": args.engine,
                   "precision": args.precision,
                   "parallelism": f"replicas x{WORLD}",
                   "l2": f"state ({bpa << n >> 20} MiB) larger than L2; no flush" if (bpa << n) > (126 << 20)
                   else "state fits L2; no flush"},
        # bytes the step's kernels read and write (each fused pass the whole
        # register once, each plain gate its changed amplitudes) per second
        "hbm_gbs": (ktimes["fused_bytes"] + ktimes["plain_bytes"]) / args.steps / sec_per_step / 1e9,
        # not an HBM rate: the bytes the one-kernel-per-gate path would move
        # for this circuit, divided by the fused step time
        "effective_gbs_plain_bytes": alg_bytes / sec_per_step / 1e9,
        "e2e": {"value": e2e_total / args.steps / WORLD, "unit": "s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(stats["kernel_launches"] / args.steps),
        "roofline": roofline,
        "fp64": fp64,
        "passes": passes,
        "step_s": per_step,
        "cpu_baseline": cpu,
        "plain": plain,
        "accuracy": accuracy,
        "planner": {"training": training, "judge": judge} if training else None,
        "clocks": clk,
    }
    if RANK == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def batch_circuits(depth, count=BATCH_CIRCUITS, seed=1):
    """The batch workload's circuits: widths uniform in 10..20 (seeded)."""
    rng = np.random.default_rng(seed)
    widths = [int(w) for w in rng.integers(10, 21, size=count)]
    return widths, [C.hea_circuit(w, depth, seed=1000 + i) for i, w in enumerate(widths)]


def batch_params(widths, depth, step):
    rng = np.random.default_rng(7919 + step)
    return rng.uniform(-math.pi, math.pi, size=sum(2 * w * depth for w in widths))


def main_batch(args, dist):
    """One step = new parameters for every circuit, one batch run, <Z_q> of
    every circuit back on the host."""
    precision = args.precision or 64
    depth = args.depth if args.depth is not None else 8
    gen, _, desc, _ = WORKLOADS["hea_batch"]
    workload = desc.format(c=args.batch_circuits, d=depth, p="complex128" if precision == 128 else "complex64")
    widths, circs = batch_circuits(depth, args.batch_circuits)
    if args.impl == "reference":
        return run_reference_batch(args, dist, widths, circs, depth, workload)
    lib = qcs_b200.Library(qcs_b200.LIB_PATH)
    b = qcs_b200.Batch(lib, precision)
    b.set_tensor_passes(args.batch_tensor)
    for w, c in zip(widths, circs):
        b.add_circuit(w, c)
    t0 = time.perf_counter()
    b.run()   # plans, tunes, captures the graph
    setup_s = time.perf_counter() - t0
    clocks = Clocks()
    clocks.start()
    for w in range(args.warmup):
        b.set_parameters(batch_params(widths, depth, w))
        b.run()
        b.expectation_z()
    barrier(dist)
    dev, wall = [], []
    for st in range(args.steps):
        params = batch_params(widths, depth, 100 + st)
        t0 = time.perf_counter()
        b.set_parameters(params)
        b.run()
        zs = b.expectation_z()
        wall.append(time.perf_counter() - t0)
        dev.append(b.info()["last_run_ms"] * 1e-3)
    barrier(dist)
    clk = clocks.stop(0)
    info = b.info()
    # accuracy: one more run with the circuits' own parameters, <Z_q> of
    # every 64th circuit against the CPU oracle (which also times them for
    # the CPU baseline)
    b.set_parameters(np.concatenate([np.asarray([v for _, p, *_ in c for v in p], dtype=np.float64)
                                     for c in circs]))
    b.run()
    z_batch = b.expectation_z()
    b.close()
    agg = aggregate_replica_times(dist, dev, WORLD)
    sec = agg["sec_per_step"]
    e2e_total = max_over_ranks(dist, sum(wall))
    peak, peak_kind = hbm_peak()
    achieved = info["pass_bytes"] / sec / 1e9
    nparams = info["parameters"]
    # the kernel that runs most passes: the batched 8x8 tensor pass or the batched register pass
    tensor_major = info["tensor_passes"] * 2 >= info["passes"]
    batch_kernel = "tensor3_pass_kernel (batched, 8x8 stages)" if tensor_major else "fused_pass_kernel (batched)"
    batch_traffic = None
    if tensor_major:
        per_amp = batch_traffic_per_amplitude()
        if per_amp is not None:
            # the measured fraction of the algorithmic bytes (complex64: 16 per amplitude and pass)
            batch_traffic = info["pass_bytes"] * per_amp / 16.0
    alg = sum(C.algorithmic_bytes(c, w, precision // 8) for w, c in zip(widths, circs))
    cpu, accuracy = None, None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu, z_oracle = cpu_baseline_batch(widths, circs, with_z=True)
        errs = [float(np.max(np.abs(z_batch[i] - z))) for i, z in z_oracle.items()]
        accuracy = {"check": f"<Z_q> of every 64th circuit ({len(errs)} circuits, all qubits) vs the CPU "
                             f"oracle (complex128), the circuits' own parameters",
                    "max_abs_err": max(errs), "tolerance": 1e-5 if precision == 64 else 1e-12}
    line = {
        "metric": f"batch wall s ({len(circs)} HEA circuits)",
        "value": agg["value"], "unit": "s", "n_gpus": WORLD, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128 (f64)" if precision == 128 else "c64 (f32 gates, f64 reductions)",
        "data": "synthetic (seeded circuits and parameters)",
        "config": {"workload": workload, "circuits": len(circs), "depth": depth, "precision": precision,
                   "tensor_passes": ["never", "tuned", "always"][args.batch_tensor],
                   "amplitudes": info["amplitudes"], "parallelism": f"replicas x{WORLD}",
                   "l2": f"registers ({info['amplitudes'] * precision // 8 >> 20} MiB) larger than L2; no flush"},
        "circuits_per_s": len(circs) / sec,
        "hbm_gbs": achieved,
        # not an HBM rate: the per-gate path's bytes over the batch step time
        "effective_gbs_plain_bytes": alg / sec / 1e9,
        "e2e": {"value": e2e_total / args.steps / WORLD, "unit": "s", "h2d_bytes_per_step": nparams * 8,
                "d2h_bytes_per_step": sum(widths) * 8},
        "gpu_launches": info["launches_per_run"],
        "roofline": {"bound": "hbm", "kernel": batch_kernel, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": f"{peak_kind} (copy, MEASURED_PEAKS hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "traffic": batch_traffic,
                     "note": "pass bytes over the whole run's device time (graph: entries in, stage matrices, "
                             "passes, <Z>, results out); traffic = DRAM bytes per run, the pass bytes scaled by "
                             "the measured bytes per amplitude of profiles/tensor3_pass_kernel_batch_traffic.txt"},
        "batch": {"groups": info["groups"], "passes": info["passes"], "tensor_passes": info["tensor_passes"],
                  "pass_bytes": info["pass_bytes"],
                  "setup_s": setup_s, "step_s": dev},
        "cpu_baseline": cpu,
        "accuracy": accuracy,
        "clocks": clk,
    }
    if RANK == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline_batch(widths, circs, stride=64, with_z=False):
    """The CPU oracle on every 64th circuit of the batch (complex128),
    scaled by 64; with_z also returns each sampled circuit's <Z_q>."""
    oracle_so = REPO / "oracle" / "liboracle_qcs.so"
    if not oracle_so.exists():
        return (None, {}) if with_z else None
    lib = qcs_b200.Library(oracle_so)
    t0 = time.perf_counter()
    count = 0
    zs = {}
    for i in range(0, len(circs), stride):
        with qcs_b200.Simulator(lib, widths[i]) as sim:
            sim.run(circs[i])
            sim.statevector()
            if with_z:
                zs[i] = sim.expectation_z()[0]
        count += 1
    dt = time.perf_counter() - t0
    cpu = {"value": dt * len(circs) / count, "unit": "s", "cores": os.cpu_count(), "kind": "port",
           "sample": f"every {stride}th circuit ({count} circuits) on the CPU oracle (complex128), {dt:.1f} s, "
                     f"scaled by {stride}"}
    return (cpu, zs) if with_z else cpu


def run_reference_batch(args, dist, widths, circs, depth, workload, stride=16):
    """The reference library, circuit by circuit through its C API (create,
    allocate, gates, one measurement of every qubit, destroy): every 16th
    circuit of the batch, scaled by 16."""
    if RANK != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    ref_so = REPO / "oracle" / "_ref" / "libqcs_ref.so"
    if not ref_so.exists():
        cpu = cpu_baseline_batch(widths, circs)
        print(json.dumps({"impl": "reference", "metric": f"batch wall s ({len(circs)} HEA circuits)",
                          "value": cpu["value"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
                          "higher_is_better": False, "config": {"workload": workload}, "cpu_baseline": cpu,
                          "e2e": {"value": cpu["value"], "unit": "s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    lib = qcs_b200.Library(ref_so)
    sample = list(range(0, len(circs), stride))
    # one simulator per register size, reset between circuits: the reference
    # sets up a communicator per simulator, so creating one per circuit does
    # not scale to thousands of circuits in one process
    sims = {}

    def step():
        for i in sample:
            n = widths[i]
            if n not in sims:
                sims[n] = qcs_b200.Simulator(lib, n, n)
            sim = sims[n]
            sim.reinitialize_mapping()
            sim.set_state("zero")
            sim.reset_clbits()
            sim.reset_measurement_state()
            sim.run(circs[i] + [("measure", (q,), (q,), (), ()) for q in range(n)])

    for _ in range(args.warmup):
        step()
    clocks = Clocks()
    clocks.start()
    wall = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        wall.append((time.perf_counter() - t0) * stride)
    clk = clocks.stop(0)
    for sim in sims.values():
        sim.close()
    value = sum(wall) / args.steps
    line = {"impl": "reference", "metric": f"batch wall s ({len(circs)} HEA circuits)", "value": value,
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)",
            "data": "synthetic (seeded circuits)",
            "config": {"workload": workload.replace("complex64", "complex128").split(" -> ")[0]
                       + " -> one measurement of every qubit, circuit by circuit (the reference has no batch, "
                         "<Z> or complex64)", "circuits": len(circs), "depth": depth},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                             "sample": f"reference library on the GPU (one simulator per register size, reset "
                                       f"between circuits), every {stride}th circuit ({len(sample)} circuits) per "
                                       f"step, host wall time scaled by {stride}"},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main_cli(args, dist):
    """The plain-method CLI workload: the driver binary (this repository's
    bin/qcs, or the reference's driver built against the reference library
    for --impl reference) runs the gate-list plug-in for every sample; one
    step = one process, timed on the host (process start to exit)."""
    n = args.qubits if args.qubits != 30 else 20
    depth = args.depth if args.depth is not None else 20
    _, _, desc, _ = WORKLOADS["cli"]
    workload = desc.format(n=n, d=depth, p="complex128")
    if RANK != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    reference = args.impl == "reference"
    exe = REPO / "oracle" / "_ref" / "qcs_ref" if reference else qcs_b200.CLI_PATH
    if not exe.exists():
        print(json.dumps({"impl": "reference" if reference else "b200", "unavailable": f"{exe} is not built"}))
        return
    circ = C.layered_u3_cz(n, depth, seed=1, measure=True)
    plug = REPO / "rqs-svg_b200" / "examples" / "gatelist.so"
    with tempfile.TemporaryDirectory() as d:
        gl = Path(d) / "circuit.txt"
        gl.write_text(C.to_gatelist(circ, n, n))
        env = dict(os.environ)
        env["QCS_GATELIST"] = str(gl)
        if not reference:
            env["QCS_FUSION"] = {"plain": "0", "greedy": "1", "learned": "2"}[args.fusion]
        cmd = [str(exe), "-s", str(CLI_SAMPLES), str(plug)]

        def step():
            t0 = time.perf_counter()
            r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
            dt = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"{exe.name} failed: {r.stderr[-500:]}")
            lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
            return dt, lines

        for _ in range(args.warmup):
            step()
        clocks = Clocks()
        clocks.start()
        wall, inside = [], []
        for _ in range(args.steps):
            dt, lines = step()
            wall.append(dt)
            inside.append(sum(ln["elapsed_time"] for ln in lines))
        clk = clocks.stop(0)
    value = sum(wall) / args.steps
    line = {"metric": f"CLI wall s, {CLI_SAMPLES} samples at {n}q", "value": value, "unit": "s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded circuit)",
            "config": {"workload": workload, "qubits": n, "depth": depth, "gates": len(circ),
                       "samples": CLI_SAMPLES, "fusion": None if reference else args.fusion},
            "samples_per_s": CLI_SAMPLES / value,
            "sum_of_sample_elapsed_s": sum(inside) / args.steps,
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk}
    if reference:
        line["impl"] = "reference"
        line["cpu_baseline"] = {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                                "sample": "the reference driver and library built from its sources for sm_100a, "
                                          "run on the GPU (it has no CPU path)"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_reference(args, dist, circuit, workload, gen, depth):
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
        line = {"impl": "reference", "metric": f"circuit wall s at {n}q ({args.workload} workload)",
                "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "c128 (f64)", "data": "synthetic (seeded circuit)",
                "config": {"workload": workload.split(" -> ")[0].replace("complex64", "complex128")
                           + " -> one measurement of every qubit (the reference has no <Z> or sampler)",
                           "qubits": n, "depth": depth, "gates": len(circuit)},
                "e2e": {"value": sum(wall) / args.steps, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                                 "sample": "reference library built from its sources for sm_100a, run on the GPU "
                                           "(it has no CPU path); host thread count 1"},
                "clocks": clk}
    else:
        cpu = cpu_baseline(gen, n, depth)
        line = {"impl": "reference", "metric": f"circuit wall s at {n}q ({args.workload} workload)",
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
