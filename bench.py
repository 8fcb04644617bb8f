"""Benchmark of the estimation epoch on B200.

One step = one estimation epoch (run_epoch) of one scenario: forward
propagation, measurement products and residuals, reference-mode derivation
and the Adam update, over all steps of every beat.

Workload (default): 20x20x20 cuboid (8,000 voxels, 24,000 states), 2,000
steps at 2 kHz, 37 triaxial sensors (111 rows), one beat, random 5^3
zero-gain block, 1% Gaussian measurement noise, Adam lr 1e-3, gains and
all-pass coefficients both trained (textbook derivative). Inputs are seeded
synthetic arrays of that shape.

Timing: W untimed warm-up epochs, then K epochs each bracketed by CUDA events
on the library's stream, with a >L2 buffer written between epochs (not
timed). Multi-GPU (torchrun): each rank runs its own scenario (different
seed), no data-path collective; time = max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "scenario-epochs/s and voxel-steps/s, chosen vs plain GPU form at stated grad tol"
UNIT = "scenario-epochs/s"
WORKLOAD = "cuboid20"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--precision", default="bf16x6", choices=["fp32", "tf32x3", "tf32", "bf16x6"],
                   help="measurement products: FP32 CUDA cores, tcgen05 3xTF32 / TF32 (guarded), tcgen05 BF16 on "
                        "error-free slices (exact accumulation)")
    p.add_argument("--batch-scenarios", type=int, default=64,
                   help="scenarios of the batched section (0 skips it)")
    p.add_argument("--batch-epochs", type=int, default=3, help="timed epochs of the batched section")
    p.add_argument("--cpu-baseline", type=int, default=1, help="time the CPU restatement's full epoch (0 skips it)")
    p.add_argument("--precision-steps", type=int, default=256,
                   help="steps of the precision report (shell, 256 triaxial sensors) against the f64 oracle (0 skips)")
    return p.parse_args()


def algorithm_config(alg):
    return alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False,
                         ap_derivative=alg.APDerivative.Textbook)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


# ----------------------------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.skip = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # the timed region starts once the sampler is producing lines (nvidia-smi takes ~0.1-0.5 s to start)
        t0 = time.perf_counter()
        while not self.lines and time.perf_counter() - t0 < 3.0:
            time.sleep(0.01)
        self.skip = len(self.lines)

    def mark(self):
        """Samples from here on count (the timed region starts)."""
        self.skip = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines[self.skip:]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------- CPU


def _cpu_epoch(scn, steps=None):
    """One oracle epoch object (f32, reference loop order) of the workload's first `steps` steps."""
    import numpy as np

    import oracle

    T = scn.num_steps if steps is None else min(steps, scn.num_steps)
    return oracle.OracleEpoch(
        scn.model.gains, scn.model.output_state_indices, scn.model.coefs, scn.model.delays,
        scn.model.initial_delays, scn.measurement_matrix, scn.control_matrix, scn.control_function[:T],
        np.ascontiguousarray(scn.measurements[:, :T]), num_batch_slots=1)


def cpu_epoch_time(scn, threads: int, steps=None):
    """Seconds of one epoch of the CPU restatement (oracle/, f32, reference loop order, bit-identical for
    any thread count) with `threads` OpenMP threads over independent outputs."""
    import oracle

    cfg = oracle.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0)
    e = _cpu_epoch(scn, steps)
    oracle.set_threads(threads)
    t0 = time.perf_counter()
    e.run_epoch(cfg)
    dt = time.perf_counter() - t0
    oracle.set_threads(0)
    return dt


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def reference_arm(args):
    """The reference's CPU epoch on the host cores: the f32 restatement of run_epoch (oracle/; the
    Rust crate cannot be built in this image), with every host core (OpenMP over independent outputs:
    results bit-identical to one thread). The K steps are one full epoch of the workload: step k is its
    time steps [k T / K, (k + 1) T / K), so the timed region is exactly one epoch and nothing is
    extrapolated (later steps run slower than early ones: decaying states become subnormal). Warm-up:
    W runs of the first T / K time steps. The reference's own threading (one thread: ndarray without
    rayon) is timed on a bounded sample, the first T / 5 steps, and reported beside it."""
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import numpy as np

    import oracle
    from cardiotrust_b200 import scenario as sc

    oracle.build()
    scn = sc.build(sc.workload_spec(args.workload, seed=0))
    t = scn.truth
    o = oracle.OracleEpoch(t.gains, t.output_state_indices, t.coefs, t.delays, t.initial_delays,
                           scn.measurement_matrix, scn.control_matrix, scn.control_function)
    y = o.simulate().astype(np.float64)
    del o
    rng = np.random.default_rng(scn.spec.seed + 7919)
    sigma = scn.spec.noise_fraction * float(np.sqrt(np.mean(y ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    cores = host_cores()
    V, T = scn.num_voxels, scn.num_steps
    seg = max(1, T // max(1, args.steps))
    for _ in range(args.warmup):
        cpu_epoch_time(scn, cores, steps=seg)
    total = cpu_epoch_time(scn, cores)
    value = 1.0 / total
    one_steps = max(1, T // 5)
    one = cpu_epoch_time(scn, 1, steps=one_steps)
    one_all = cpu_epoch_time(scn, cores, steps=one_steps)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{args.workload}: 20x20x20 cuboid, {V} voxels, {3 * V} states, T={T}, "
                               f"{scn.num_sensors} sensor rows, 1 beat, 1 % noise, Adam lr 1e-3, gains+coefficients",
                   "parallelism": f"{cores} host threads (OpenMP over independent outputs)",
                   "step": f"time steps [k T/K, (k+1) T/K) of one epoch ({seg} of {T})"},
        "voxel_steps_per_s": value * V * T,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"one full {T}-step epoch ({total:.1f} s) timed as {args.steps} steps; "
                                   f"{args.warmup} warm-up runs of the first {seg} time steps",
                         "single_thread_sample": {
                             "seconds": one, "cores": 1, "threads_speedup_on_sample": one / one_all,
                             "sample": f"first {one_steps} of {T} time steps (before states decay to subnormal "
                                       f"values; the full all-core epoch above includes the slower later steps)"}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------------------- GPU


def profiled_counters(kernel, workload):
    """Per-launch ncu figures of `kernel` on `workload` from its committed summary
    (profiles/<kernel>_<workload>.md): DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum), warp
    instructions, and the capture date and file, or None where the summary lacks them."""
    import re

    path = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not path.exists():
        return None
    text = path.read_text()
    out = {"file": f"profiles/{path.name}"}
    for key, pat in (("traffic", r"^traffic_bytes_per_launch:\s*(\d+)"),
                     ("instructions", r"^warp_instructions_per_launch:\s*(\d+)"),
                     ("date", r"^captured:\s*(\S+)")):
        m = re.search(pat, text, re.M)
        out[key] = (int(m.group(1)) if key != "date" else m.group(1)) if m else None
    return out


def timed_epochs(stream, run, n, flush=None):
    """Device time (ms) of `n` calls of `run`, each bracketed by CUDA events on `stream`."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    for k in range(n):
        if flush is not None:
            flush.random_(0, 255)
        ev[k][0].record(stream)
        run()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def forms_section(alg, eng, bi, prec, stream, flush, scn):
    """The plain GPU form and the adjoint mode on the headline workload."""
    V, T, B = scn.num_voxels, scn.num_steps, scn.num_beats
    out = {}
    # these epochs reuse batch-metric slot 0: only their timing is read
    eng.run_epoch_plain(0, sync=True)  # warm-up (allocates the plain form's buffers)
    l0 = eng.kernel_launches()
    ms = timed_epochs(stream, lambda: eng.run_epoch_plain(0, sync=False), 2, flush)
    eng.sync()
    launches = (eng.kernel_launches() - l0) // 2
    out["plain"] = {"form": "plain GPU form: one launch per phase per step (reference gradients, FP32)",
                    "scenario_epochs_per_s": 1000.0 / statistics.mean(ms), "ms_per_epoch": statistics.mean(ms),
                    "voxel_steps_per_s": V * T * B * 1000.0 / statistics.mean(ms), "launches_per_epoch": int(launches)}
    eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec, sync=True)
    eng.set_profiling(True)
    ms = timed_epochs(stream, lambda: eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec, sync=False),
                      3, flush)
    prof = eng.read_profile()
    eng.set_profiling(False)
    out["adjoint"] = {"form": "persistent kernels, adjoint gradients (checkpoints every 256 steps)",
                      "scenario_epochs_per_s": 1000.0 / statistics.mean(ms), "ms_per_epoch": statistics.mean(ms),
                      "voxel_steps_per_s": V * T * B * 1000.0 / statistics.mean(ms),
                      "phase_ms": {k: v[0] / 3 for k, v in prof.items() if v[0] > 0}}
    return out


def post_run_section(alg, eng, scn, stream, hbm_peak, prec):
    """The callers either side of the epoch on the headline workload: the post-run pass (spherical
    arrays of the last beat, their maxima, activation times; then the 101-threshold segmentation
    metrics) and the reference's epoch loop (learning-rate schedule, per-epoch summary read-back)."""
    import torch

    V, T = scn.num_voxels, scn.num_steps
    sr = scn.spec.sample_rate_hz
    eng.calculate_plotting_arrays(sr)
    ms = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.calculate_plotting_arrays(sr)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    call_ms = min(ms)
    algo_bytes = 24.0 * T * V  # 12 B of states read and 12 B of magnitude/theta/phi written per (step, voxel)
    achieved = algo_bytes / (call_ms / 1000.0) / 1e9
    t0 = time.perf_counter()
    fm = eng.calculate_final(scn.types_truth, scn.numbers)
    first_ms = (time.perf_counter() - t0) * 1000.0  # includes the one-time buffer set-up and kernel loading
    fms = []
    for _ in range(5):
        t0 = time.perf_counter()
        fm = eng.calculate_final(scn.types_truth, scn.numbers)
        fms.append((time.perf_counter() - t0) * 1000.0)
    final_ms = min(fms)
    model = model_construction(alg, eng, scn)
    loop_epochs = 5
    a = dataclasses.replace(algorithm_config(alg), epochs=loop_epochs, learning_rate_reduction_interval=2,
                            learning_rate_reduction_factor=0.5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # batch-metric slots from 0 again: only the timing and the epoch count are read
    summ, _, _ = eng.run_model_based(0, precision=prec, algorithm=a)
    loop_s = time.perf_counter() - t0
    return {
        "plotting_arrays": {"call_ms": call_ms, "algorithmic_bytes": algo_bytes, "achieved_gbs": achieved,
                            "frac": achieved / hbm_peak,
                            "note": "CUDA events around the synchronous C call (its device sync included)"},
        "final_metrics": {"call_ms": final_ms, "first_call_ms": first_ms, "threshold": fm.threshold,
                          "dice": fm.dice, "iou": fm.iou,
                          "note": "wall clock of the C call (best of 5 after the first): grid upload, states scan, "
                                  "threshold sweep, read-back"},
        "model_construction": model,
        "scenario_loop": {"epochs": loop_epochs, "epochs_run": summ["epochs_run"],
                          "scenario_epochs_per_s": loop_epochs / loop_s,
                          "note": "ct_run_model_based wall clock: schedule, one summary read-back per epoch"},
    }


def model_construction(alg, eng, scn):
    """The step before the epoch on the headline workload: the Biot-Savart measurement matrix and the
    delay arrays built on the device (wall clock of the synchronous C calls, best of 5 after the
    first) against the host builder's vectorised numpy restatement of the same loops."""
    import numpy as np

    from cardiotrust_b200 import scenario as sc

    spec = scn.spec
    sd = alg.SpatialDescription.from_scenario(scn)

    def best(fn, n=5):
        fn()
        ts = []
        for _ in range(n):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1000.0)
        return min(ts)

    fill_ms = best(lambda: eng.set_measurement_matrix(sd))
    h_ms = best(lambda: alg.measurement_matrix(eng.ctx, sd))
    d_ms = best(lambda: alg.delay_samples(eng.ctx, sd))
    host_h_ms = best(lambda: sc._measurement_matrix(spec, scn.types_model, scn.numbers, scn.positions_mm,
                                                    scn.sensor_positions_mm, scn.sensor_orientations), n=2)
    host_d_ms = best(lambda: sc._delay_samples(scn.types_model, scn.numbers, scn.positions_mm, spec.velocity_m_per_s,
                                               spec.sample_rate_hz), n=2)
    H = alg.measurement_matrix(eng.ctx, sd)
    samples, delays, coefs = alg.delay_samples(eng.ctx, sd)
    same = bool(np.array_equal(H, scn.measurement_matrix) and np.array_equal(samples, scn.model.initial_delays)
                and np.array_equal(delays, scn.model.delays) and np.array_equal(coefs, scn.model.coefs))
    return {"lead_field_into_scenario_ms": fill_ms, "lead_field_to_host_ms": h_ms, "delay_arrays_to_host_ms": d_ms,
            "host_builder_lead_field_ms": host_h_ms, "host_builder_delays_ms": host_d_ms,
            "bit_identical_to_host_builder": same, "matrix_bytes": int(H.nbytes),
            "note": "wall clock of the synchronous C calls (uploads, kernel, operand splits or read-back)"}


def _noisy_scenario(alg, sc, ctx, spec):
    """A batch-workload scenario with its ground truth from the CUDA forward plus the spec's noise."""
    import numpy as np

    scn = sc.build(spec, ctx=ctx)
    truth = alg.EpochEngine.from_scenario(ctx, scn, truth=True)
    y = truth.simulate()
    truth.close()
    rng = np.random.default_rng(spec.seed + 7919)
    sigma = spec.noise_fraction * float(np.sqrt(np.mean(y.astype(np.float64) ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    return scn


def batch_precision_check(alg, sc, ctx, specs, work, prec):
    """Gradient error of the batched epoch's product precision on members of the batch workload, one
    adjoint epoch from the initial parameters (beats in index order, as in the batch): the smallest,
    median and largest members against the same epoch with FP32 products (which the precision report
    places within ~1.5e-4 of the f64 oracle), and the smallest member with its beat cut to 600 steps
    against the f64 oracle's adjoint gradient (the oracle needs ~20 s per 3,000-step beat of it)."""
    import dataclasses

    import numpy as np

    import oracle

    def rel(a, b):
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))

    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False,
                        ap_derivative=alg.APDerivative.Textbook)

    def gpu_grads(scn, precision):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        eng.run_epoch(0, beat_order=np.arange(scn.num_beats), grad_mode=alg.GradMode.Adjoint, precision=precision)
        g = (eng.read("grad_gains"), eng.read("grad_coefs"))
        eng.close()
        return g

    def entry(i, scn, against, got, ref):
        return {"member": int(i), "voxels": scn.num_voxels, "steps": scn.num_steps, "beats": scn.num_beats,
                "states_multiple_of_4": scn.num_states % 4 == 0, "against": against,
                "grad_gains": rel(got[0], ref[0]), "grad_coefs": rel(got[1], ref[1])}

    order = np.argsort(work)
    out = {"target": 1e-3, "members": []}
    for i in (order[0], order[len(order) // 2], order[-1]):
        scn = _noisy_scenario(alg, sc, ctx, specs[int(i)])
        out["members"].append(entry(i, scn, "GPU epoch with FP32 products", gpu_grads(scn, prec),
                                    gpu_grads(scn, alg.Precision.Fp32)))
    i = order[0]
    scn = _noisy_scenario(alg, sc, ctx, dataclasses.replace(specs[int(i)], num_steps=600))
    o = oracle.from_scenario(scn, dtype=np.float64)
    o.run_epoch(oracle.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0, ap_derivative=1),
                beat_order=np.arange(scn.num_beats, dtype=np.int32), adjoint=True)
    out["members"].append(entry(i, scn, "f64 oracle adjoint (beat cut to 600 steps)", gpu_grads(scn, prec),
                                (o.d_gains, o.d_coefs)))
    out["max"] = max(max(m["grad_gains"], m["grad_coefs"]) for m in out["members"])
    return out


def batched_section(args, alg, sc, ctx, prec, stream, flush, rank=0, world=1):
    """64 scenarios of uneven size (batch_workload_specs): the batched adjoint epoch (one forward and
    one adjoint launch per beat index over every member, replayed from a CUDA graph) against the plain
    one-scenario GPU form run over every member in turn, and against the persistent one-scenario
    adjoint epoch (ct_run_epoch) run over every member in turn. With N ranks the scenarios are split
    by a greedy balance of voxel-steps (replicas.shard_scenarios), each rank batches its share, and
    every time is the max over ranks; no collective touches the data path."""
    import numpy as np

    from cardiotrust_b200 import replicas

    t0 = time.perf_counter()
    all_specs = sc.batch_workload_specs(args.batch_scenarios, seed=0)
    costs = [replicas.scenario_cost(sc.voxel_count(sp), sp.num_steps, sp.num_beats) for sp in all_specs]
    mine = replicas.shard_scenarios(costs, world)[rank]
    specs = [all_specs[i] for i in mine]
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False,
                        ap_derivative=alg.APDerivative.Textbook)
    engines, vtb, sizes, vtbs = [], 0, [], []
    slots = 2 + 5 + args.batch_epochs + 1 + 2  # warm-up, autotuner trials, timed and profiled epochs, plain
    for sp in specs:
        scn = _noisy_scenario(alg, sc, ctx, sp)
        engines.append(alg.EpochEngine.from_scenario(ctx, scn, num_batch_slots=slots, algorithm=cfg))
        vtb += scn.num_voxels * scn.num_steps * scn.num_beats
        vtbs.append(scn.num_voxels * scn.num_steps * scn.num_beats)
        sizes.append(scn.num_voxels)
        del scn
    build_s = time.perf_counter() - t0
    batch = alg.EpochBatch(ctx, engines, grad_mode=alg.GradMode.Adjoint, precision=prec)
    batch.run_epoch(sync=True)  # warm-up: captures the epoch graph
    tuned = batch.autotune()    # up to five trial epochs (they train); keeps the fastest schedule
    batch.run_epoch(sync=True)  # captures the tuned schedule
    ms = timed_epochs(stream, lambda: batch.run_epoch(sync=False), args.batch_epochs, flush)
    batch.sync()
    info = batch.info()
    # one more epoch as eager launches with CUDA events around each phase (where the epoch goes)
    batch.set_profiling(True)
    batch.run_epoch(sync=True)
    phases = {k: v for k, v in batch.read_profile().items() if v > 0}
    batch.set_profiling(False)
    chosen_ms = replicas.max_over_ranks(statistics.mean(ms))
    n = len(all_specs)
    vtb = int(replicas.sum_over_ranks(vtb))
    # the persistent one-scenario adjoint epoch (ct_run_epoch) over every member in turn, same products
    small = int(np.argmin(sizes))
    engines[small].run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec, sync=True)
    seq_ms = 0.0
    for e in engines:
        seq_ms += timed_epochs(stream, lambda: e.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec,
                                                             sync=False), 1, flush)[0]
    seq_ms = replicas.max_over_ranks(seq_ms)
    # plain one-scenario form over every member, one epoch each (after one warm-up epoch of the smallest)
    engines[small].run_epoch_plain(0, sync=True)
    plain_ms = 0.0
    for k, e in enumerate(engines):
        plain_ms += timed_epochs(stream, lambda: e.run_epoch_plain(0, sync=False), 1)[0]
    plain_ms = replicas.max_over_ranks(plain_ms)
    batch.close()
    for e in engines:
        e.close()
    check = batch_precision_check(alg, sc, ctx, specs, vtbs, prec) if world == 1 else None
    chosen = n * 1000.0 / chosen_ms
    plain = n * 1000.0 / plain_ms
    seq = n * 1000.0 / seq_ms
    return {
        "workload": f"{n} scenarios: voxels log-uniform 500..30000 (cuboids and shells), 1-8 beats, 1000-4000 "
                    "steps, 37-128 triaxial sensors, random 3^3 pathological block and pulse onset, Adam lr 1e-3, "
                    "gains+coefficients",
        "scenarios": n, "ranks": world, "scenarios_this_rank": len(specs),
        "voxels_total_this_rank": int(sum(sizes)), "voxel_steps_per_epoch": int(vtb),
        "build_s": build_s,
        "chosen": {"form": "batched: one persistent forward and one persistent adjoint launch per beat index over "
                           "every member's tiles, epoch replayed from a CUDA graph; adjoint gradients, checkpoint interval "
                           "from the autotuner", "precision": f"{['fp32', 'tf32x3', 'tf32', 'bf16x6'][int(prec)]} products for every member",
                   "scenario_epochs_per_s": chosen, "voxel_steps_per_s": vtb * 1000.0 / chosen_ms,
                   "ms_per_epoch": chosen_ms, "graph_kernels": info["graph_kernels"], "uses_graph": info["uses_graph"],
                   "forward_ctas": info["forward_ctas"], "adjoint_ctas": info["adjoint_ctas"], "autotuned": tuned,
                   "eager_phase_ms": phases},
        "plain": {"form": "plain GPU form, one scenario at a time, one launch per phase per step (reference "
                          "gradients, FP32)", "scenario_epochs_per_s": plain,
                  "voxel_steps_per_s": vtb * 1000.0 / plain_ms, "ms_per_epoch_all": plain_ms},
        "sequential_persistent": {"form": "the persistent one-scenario adjoint epoch (ct_run_epoch), one member "
                                          "after another, same products", "scenario_epochs_per_s": seq,
                                  "voxel_steps_per_s": vtb * 1000.0 / seq_ms, "ms_per_epoch_all": seq_ms},
        "chosen_vs_plain": chosen / plain,
        "chosen_vs_sequential_persistent": chosen / seq,
        "gradient_error": check,
    }


def precision_reference(workload, steps):
    """One precision-report case and its f64 oracle results (run on the host, in a thread).

    The workload (the precision config: the 64x64x48 shell with 256 triaxial sensors = 768 rows; or
    the headline cuboid) with its beat cut to `steps` steps, so that the f64 CPU oracle finishes in
    tens of seconds; ground truth from the f32 oracle forward plus the workload's 1 % noise. Returns
    (scenario, {name: f64 result}) of one reference-mode epoch and of the adjoint gradient, both from
    the pre-update parameters."""
    import numpy as np

    import oracle
    from cardiotrust_b200 import scenario as sc

    spec = sc.workload_spec(workload)
    spec.num_steps = steps
    scn = sc.build(spec)
    t = scn.truth
    fwd = oracle.OracleEpoch(t.gains, t.output_state_indices, t.coefs, t.delays, t.initial_delays,
                             scn.measurement_matrix, scn.control_matrix, scn.control_function)
    y = fwd.simulate().astype(np.float64)
    del fwd
    rng = np.random.default_rng(spec.seed + 7919)  # 1 % noise, as the precision config specifies
    sigma = spec.noise_fraction * float(np.sqrt(np.mean(y ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    a = oracle.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0)
    ref = oracle.from_scenario(scn, dtype=np.float64)
    ref.run_epoch(a)
    out = {"system_states": ref.system_states.copy(), "measurements": ref.measurements.copy(),
           "residuals": ref.residuals.copy(), "grad_gains": ref.d_gains.copy(), "grad_coefs": ref.d_coefs.copy()}
    del ref
    adj = oracle.from_scenario(scn, dtype=np.float64)
    adj.stated_loss(a, gradient=True)
    out["adjoint_grad_gains"] = adj.d_gains.copy()
    out["adjoint_grad_coefs"] = adj.d_coefs.copy()
    del adj
    # the reference's own arithmetic: the f32 restatement (reference loop order) against the same f64
    def rel(x, y):
        y = np.asarray(y, np.float64)
        return float(np.linalg.norm(np.asarray(x, np.float64) - y) / max(np.linalg.norm(y), 1e-300))

    f32 = oracle.from_scenario(scn)
    f32.run_epoch(a)
    f32_err = {k: rel(v, out[k]) for k, v in (("system_states", f32.system_states), ("measurements", f32.measurements),
                                               ("residuals", f32.residuals), ("grad_gains", f32.d_gains),
                                               ("grad_coefs", f32.d_coefs))}
    del f32
    f32 = oracle.from_scenario(scn)
    f32.run_epoch(a, adjoint=True)
    f32_err["adjoint_grad_gains"] = rel(f32.d_gains, out["adjoint_grad_gains"])
    f32_err["adjoint_grad_coefs"] = rel(f32.d_coefs, out["adjoint_grad_coefs"])
    out["f32_reference"] = f32_err
    return scn, out


PRECISION_CASES = (("shell_precision", None), ("cuboid20", 400))


def precision_cases(steps):
    return [precision_reference(w, steps if n is None else n) for w, n in PRECISION_CASES]


def precision_section(alg, ctx, job):
    """Relative error (norm-wise, f64) of every result of each product precision against the f64 oracle."""
    job.join()
    if job.error is not None:
        return {"error": repr(job.error)}
    out = {"error": "||gpu - f64 oracle|| / ||f64 oracle|| per result (states [T,S], measurements [T,M], last-step "
                    "residuals, reference-mode and adjoint gradients)",
           "targets": {"states": 1e-4, "gradients": 1e-3}, "cases": []}
    for scn, ref in job.result:
        out["cases"].append(precision_case(alg, ctx, scn, ref))
    return out


def precision_case(alg, ctx, scn, ref):
    import numpy as np

    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)

    def rel(a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    from cardiotrust_b200 import _lib

    results = {}
    for name, prec in (("fp32", alg.Precision.Fp32), ("tf32x3", alg.Precision.Tf32x3), ("tf32", alg.Precision.Tf32),
                       ("bf16x6", alg.Precision.Bf16x6)):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        try:
            eng.run_epoch(0, beat_order=np.arange(scn.num_beats), precision=prec)
        except _lib.CtError as exc:  # the library's guard of the TF32 modes
            eng.close()
            results[name] = {"refused": str(exc)}
            continue
        r = {f: rel(eng.read(f), ref[f]) for f in ("system_states", "measurements", "residuals", "grad_gains",
                                                   "grad_coefs")}
        eng.close()
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        eng.run_epoch(0, beat_order=np.arange(scn.num_beats), grad_mode=alg.GradMode.Adjoint, precision=prec)
        r["adjoint_grad_gains"] = rel(eng.read("grad_gains"), ref["adjoint_grad_gains"])
        r["adjoint_grad_coefs"] = rel(eng.read("grad_coefs"), ref["adjoint_grad_coefs"])
        eng.close()
        results[name] = r
    results["f32_reference_restatement (CPU, reference loop order)"] = ref["f32_reference"]
    return {
        "workload": f"{scn.spec.mask} {scn.spec.shape} ({scn.num_voxels} voxels, {scn.num_states} states), "
                    f"{scn.num_sensors} sensor rows, beat cut to {scn.num_steps} steps so the f64 CPU oracle "
                    "finishes; 1 % noise; Adam, gains+coefficients",
        "results": results,
    }


class _Job(threading.Thread):
    def __init__(self, fn, *a):
        super().__init__(daemon=True)
        self.fn, self.a, self.result, self.error = fn, a, None, None

    def run(self):
        try:
            self.result = self.fn(*self.a)
        except Exception as exc:  # reported in the JSON line, never fatal
            self.error = exc


def gpu_arm(args):
    import numpy as np
    import torch

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    from cardiotrust_b200 import algorithm as alg
    from cardiotrust_b200 import scenario as sc

    # a dedicated stream: the library issues every kernel on it, and the timing events,
    # the L2 flush and the barriers below are ordered on it too
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = alg.Context(local_rank, stream=stream.cuda_stream)
    scn = sc.build(sc.workload_spec(args.workload, seed=rank), ctx=ctx)
    # ground truth with the CUDA forward (Simulation::run reuses the prediction path)
    truth = alg.EpochEngine.from_scenario(ctx, scn, truth=True)
    y = truth.simulate()
    truth.close()
    rng = np.random.default_rng(scn.spec.seed + 7919)
    sigma = scn.spec.noise_fraction * float(np.sqrt(np.mean(y.astype(np.float64) ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)

    cfg = algorithm_config(alg)
    prec = {"fp32": alg.Precision.Fp32, "tf32x3": alg.Precision.Tf32x3, "tf32": alg.Precision.Tf32,
            "bf16x6": alg.Precision.Bf16x6}[args.precision]
    total_epochs = args.warmup + 3 * args.steps + 4
    eng = alg.EpochEngine.from_scenario(ctx, scn, num_batch_slots=total_epochs, algorithm=cfg)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    V, T, B = scn.num_voxels, scn.num_steps, scn.num_beats

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    bi = 0
    for _ in range(args.warmup):
        bi = eng.run_epoch(bi, precision=prec, sync=True)
    barrier()

    # ---- device-resident timed region (clock samples every 50 ms from here to its end)
    launches0 = eng.kernel_launches()
    clocks.mark()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.random_(0, 255)
        ev[k][0].record(stream)
        bi = eng.run_epoch(bi, precision=prec, sync=False)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    eng.sync()
    clock = clocks.stop()
    launches = (eng.kernel_launches() - launches0) // args.steps
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(ms)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1000.0)
    barrier()

    # ---- end to end through the C ABI with host buffers (pinned), copies inside the timed region
    # the model and the measurements in pinned host memory, as a Rust caller of run_epoch holds them:
    # ct_run_epoch_host copies them in, runs the epoch and copies the updated parameters and the
    # batch-wise loss back into the same buffers, waiting once
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_gains, h_coefs = pin(eng.read("gains")), pin(eng.read("coefs"))
    h_delays, h_meas = pin(eng.read("delays")), pin(scn.measurements)
    out_loss = pin(np.empty(eng.dims["NB"], np.float32))
    h2d = h_gains.nbytes + h_coefs.nbytes + h_delays.nbytes + h_meas.nbytes
    d2h = h_gains.nbytes + h_coefs.nbytes + h_delays.nbytes + out_loss.nbytes
    e2e_steps = max(3, args.steps // 2)
    bi = eng.run_epoch_host(bi, h_gains, h_coefs, h_delays, h_meas, out_loss, precision=prec)  # allocates staging
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        bi = eng.run_epoch_host(bi, h_gains, h_coefs, h_delays, h_meas, out_loss, precision=prec)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * e2e_steps / e2e_s
    barrier()

    # ---- per-phase device time (CUDA events on the library stream) for the roofline
    eng.set_profiling(True)
    for _ in range(args.steps):
        flush.random_(0, 255)
        bi = eng.run_epoch(bi, precision=prec, sync=False)
    prof = eng.read_profile()
    eng.set_profiling(False)
    peaks = {}
    pp = ROOT / "MEASURED_PEAKS.json"
    if pp.exists():
        peaks = json.loads(pp.read_text())
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    S = 3 * V
    phase_ms = {k: v[0] / args.steps for k, v in prof.items()}
    # the dominant kernel of the epoch is the forward propagation (one launch per beat)
    launches_of = max(1, prof["forward"][1] // args.steps)
    per_launch_ms = phase_ms["forward"] / launches_of
    # the resident form runs when every 32-voxel tile fits a co-resident CTA (two per SM)
    fwd_kernel = "forward_ring_kernel" if (V + 31) // 32 <= 2 * 148 else "forward_stream_kernel"
    # bytes a launch must move through HBM in this design: the state history it writes (4 B per
    # state-step), and once per launch the gains [S,78], coefficients, delays and neighbour table
    # [V,26], the all-pass state [V,78] read and written, control column and function
    must = 4.0 * S * T + 4.0 * 78 * S + 12.0 * 26 * V + 2 * 4.0 * 78 * V + 4.0 * S + 4.0 * T
    achieved = must / (per_launch_ms / 1000.0) / 1e9
    pc = profiled_counters(fwd_kernel, args.workload) or {}
    sm_mhz = (clock or {}).get("sm_mhz") or 1965.0
    issue = None
    if pc.get("instructions"):
        issue = pc["instructions"] / (148 * 4 * sm_mhz * 1e6 * per_launch_ms / 1000.0)
    roofline = {"bound": "hbm", "kernel": fwd_kernel, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_source": peak_src,
                "traffic": pc.get("traffic"),
                "traffic_source": (f"{pc['file']} (ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                   f"captured {pc.get('date')})") if pc else None,
                "algorithmic_bytes_per_launch": must,
                "algorithmic_model": "state history written once (4 B per state-step) + per-launch parameters "
                                     "and all-pass state; neighbour history, gains and chain state stay on chip",
                "launch_ms": per_launch_ms,
                "limiter": "issue and latency, not HBM: warp-instruction issue over the SMs' 4 schedulers at the "
                           "median SM clock is `issue_utilisation`; the step recurrence serialises time",
                "issue_utilisation": issue,
                "reference_layout_throughput": {
                    "bytes_per_state_step": 601, "GB_per_s": 601.0 * S * T / (per_launch_ms / 1000.0) / 1e9,
                    "note": "the reference's per-step reads (gains, all-pass state, coefficients, history every step) "
                            "over the launch time: a throughput figure, not HBM traffic"}}

    # ---- plain GPU form and adjoint mode on the same workload; the batched workload. The plain forms
    # are launch-bound, so nothing else runs on the host while they are timed.
    forms = forms_section(alg, eng, bi, prec, stream, flush, scn)
    post_run = post_run_section(alg, eng, scn, stream, hbm_peak, prec)
    batched = None
    if args.batch_scenarios > 0:
        eng.close()
        batched = batched_section(args, alg, sc, ctx, prec, stream, flush, rank, world)

    # ---- precision report: the f64 oracle on the host, then the GPU products of the same cases
    precision = None
    if args.precision_steps > 0 and rank == 0 and world == 1:
        prec_job = _Job(precision_cases, args.precision_steps)
        prec_job.start()
        precision = precision_section(alg, ctx, prec_job)

    # ---- CPU baseline (rank 0, N = 1 only): one full epoch of the CPU restatement on every host core
    cpu = None
    if rank == 0 and world == 1 and args.cpu_baseline:
        try:
            import oracle

            oracle.build()
            cores = host_cores()
            dt = cpu_epoch_time(scn, cores)
            cpu = {"value": 1.0 / dt, "unit": UNIT, "cores": cores, "kind": "port",
                   "sample": f"one full {T}-step epoch of the workload ({dt:.1f} s), f32 restatement in the "
                             "reference's loop order, OpenMP over independent outputs (bit-identical to one thread)"}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"fp32": "f32", "tf32x3": "f32 (products tf32x3)", "tf32": "f32 (products tf32)",
                      "bf16x6": "f32 (products bf16x6: BF16 slices, exact FP32 accumulation)"}[args.precision],
            "data": "synthetic (seeded)",
            "config": {
                "workload": f"{args.workload}: 20x20x20 cuboid, {V} voxels, {S} states, T={T}, "
                            f"{scn.num_sensors} sensor rows, {B} beat, Adam lr 1e-3, gains+coefficients (textbook)",
                "voxels": V, "states": S, "steps_per_epoch": T, "beats": B, "sensor_rows": scn.num_sensors,
                "grad_mode": "reference", "precision": args.precision,
                "l2": "256 MB buffer written between timed epochs (not timed)",
                "parallelism": f"replicas x{world}",
            },
            "voxel_steps_per_s": value * V * T * B,
            "phase_ms": phase_ms,
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "call": "ct_run_epoch_host: gains, coefficients, delays and measurements copied in from pinned "
                            "host memory, updated parameters and batch-wise loss copied out, every epoch"},
            "clocks": clock,
            "forms": forms,
            "chosen_vs_plain": value / forms["plain"]["scenario_epochs_per_s"],
            "batched": batched,
            "post_run": post_run,
            "precision": precision,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
