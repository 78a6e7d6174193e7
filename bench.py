"""Benchmark: spin-factorized H.v throughput on the 4x4 Hubbard cluster.

Workload: 4x4 open square cluster, t=-1, t'=0.3, U=8, half filling
(sector R0:N16:S0, dimension 12870^2 = 165,636,900; one FP64 vector = 1.33 GB).
One step = one application y = H x of the solver's device Hamiltonian to an
HBM-resident vector (the operation the Lanczos and band-Lanczos recurrences
repeat). Metric: H.v algorithmic HBM throughput, 16 bytes per basis state per
application (read x once, write y once); inputs are 1.33 GB, larger than L2,
so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--solve]

N > 1 runs one replica per GPU (launched by torch.distributed.run); the line
reports the aggregate of all replicas, timed as the max over ranks.
--impl reference times the reference's own CPU H.v (Hamiltonian_Factorized::mult_add,
compiled from its sources in oracle/_ref) on the same sector.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H.v HBM GB/s"
UNIT = "GB/s"
WORKLOAD = "4x4 Hubbard cluster (open, t=-1, t'=0.3, U=8, half filling, sector R0:N16:S0, dim 165636900)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solve", action="store_true", help="time the full 4x4 solve also for N > 1")
    ap.add_argument("--no-solve", action="store_true",
                    help="skip the full 4x4 ground state + Green function timed by default at N = 1")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the batched-solve metrics reported beside the H.v line")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: warm-up and timed H.v only (no e2e, clocks or CPU baseline)")
    ap.add_argument("--sector", default=None, help="sector of the 4x4 cluster to use (default R0:N16:S0)")
    ap.add_argument("--hv-windows", action="store_true",
                    help="with --profile: H.v through the window kernels (option hv_windows) instead of the "
                         "staged ones")
    ap.add_argument("--workload", default="hv", choices=["hv", "batch", "baths", "vca", "cdmft"],
                    help="hv: H.v on the 4x4 cluster (default); batch: independent random clusters, "
                         "every sector, ground state + Green function; baths: 2x2 + 8-bath points; "
                         "vca: 2x5-cluster VCA, surrogate-guided against ED-only")
    ap.add_argument("--vca-points", type=int, default=4096, help="training points of the VCA surrogate")
    ap.add_argument("--vca-epochs", type=int, default=400, help="training epochs of the VCA surrogate")
    ap.add_argument("--batch", type=int, default=64, help="instances per step for --workload batch/baths")
    ap.add_argument("--threads", type=int, default=0, help="host threads for batched solves (0 = all)")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if (args.impl == "ours" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(values, world, device="cpu"):
    """Element-wise max of per-rank timings (the slowest replica sets the step time)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def aggregate_value(bytes_per_step, ms_per_step, world):
    """Whole-job throughput in GB/s: every replica processed bytes_per_step per step."""
    return world * bytes_per_step / (ms_per_step * 1e-3) / 1e9


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one H.v, one
# k_hv_cols16w launch (writes y = dn hops x) and one k_hv_rows16 launch (adds the
# up hops and the diagonal, reads y back), per basis state: ncu --set full on the
# 4x4 N_up = N_dn = 6 sector (64,128,064 states, vectors larger than L2) read
# 0.983 + 1.511 GB (profiles/hv_staged_sq4x4_N12_ncu_full.md). Both passes stream
# the vectors once, so the traffic scales with the number of states.
TRAFFIC_BYTES_PER_STATE = (0.514972e9 + 0.467877e9 + 1.029826e9 + 0.481437e9) / 64128064


def ncu_traffic(D):
    return TRAFFIC_BYTES_PER_STATE * D


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "100"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


class UtilSampler:
    """Mean GPU utilization (nvidia-smi utilization.gpu, the fraction of time a
    kernel was running) sampled every 100 ms while a step runs."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=utilization.gpu", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "100"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        vals = []
        with open(self.file.name) as f:
            for line in f:
                try:
                    vals.append(float(line.strip()))
                except ValueError:
                    pass
        os.unlink(self.file.name)
        return {"mean_pct": statistics.mean(vals), "samples": len(vals)} if vals else None


def cpu_baseline_sample():
    """The reference's mult_add on the same sector, one application, one core."""
    from oracle import ref
    from pyqcm_b200 import workloads as W
    p = W.square4x4()
    ref.load_problem(p, 9001, model_name="bench_ref_sq4x4", fmt="F")
    H = ref.RefHamiltonian(9001, p.sectors)
    return H


def run_reference(args, world, rank):
    if rank != 0:
        return
    H = cpu_baseline_sample()
    D = H.dim
    steps, warm = max(1, min(args.steps, 3)), min(args.warmup, 1)
    for _ in range(warm):
        H.bench(1)
    t0 = time.perf_counter()
    for _ in range(steps):
        H.bench(1)
    dt = (time.perf_counter() - t0) / steps
    v = 16.0 * D / dt / 1e9
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "steps_requested": args.steps, "warmup_requested": args.warmup,
            "steps_capped": (f"ran {steps} timed step(s) and {warm} warm-up step(s) of the {args.steps} + "
                             f"{args.warmup} requested: one H.v of the reference on one core takes "
                             f"{dt:.1f} s") if (steps, warm) != (args.steps, args.warmup) else None,
            "config": {"workload": WORKLOAD, "inputs": "larger than L2 (1.33 GB vectors)",
                       "reference": "Hamiltonian_Factorized::mult_add compiled from the reference sources (oracle/_ref)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{steps} full H.v application(s) of the 4x4 sector; the reference's H.v has no threading"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if world == 1 and not args.no_secondary:
        line["secondary"] = secondary_lines("reference")
        line.update(secondary_summary(line["secondary"]))
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch

    import pyqcm_b200 as qed
    from pyqcm_b200 import workloads as W
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    qed.init(local)
    prob = W.square4x4()
    if args.sector:
        prob.sectors = args.sector
    label = 7000 + rank
    qed.load_problem(prob, label, model_name="bench_sq4x4", fmt="F")
    if args.hv_windows:
        if not args.profile:
            raise SystemExit("--hv-windows is a profiling switch: use it with --profile")
        qed.set_global_parameter("hv_windows", True)
    H = qed.Hamiltonian(label, prob.sectors)
    D = H.dim
    g = torch.Generator(device=f"cuda:{local}").manual_seed(1234 + rank)
    x = torch.randn(D, dtype=torch.float64, device=f"cuda:{local}", generator=g)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        H.apply_device(x.data_ptr(), y.data_ptr(), sh)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        H.apply_device(x.data_ptr(), y.data_ptr(), sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "dim": D, "ms_per_hv": ms,
                              "GBps_16D": 16.0 * D / (ms * 1e-3) / 1e9,
                              "window_launches": qed.window_launches(),
                              "hv_tuning": qed.hv_tuning_report()}), flush=True)
        return
    # end to end through the C ABI with host buffers (y += H x, copies inside)
    xh = torch.empty(D, dtype=torch.float64, pin_memory=True).numpy()
    yh = torch.empty(D, dtype=torch.float64, pin_memory=True).numpy()
    xh[:] = x.cpu().numpy()
    yh[:] = 0.0
    H.mult_add(xh, yh)  # warm-up
    e2e_steps = 3
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        H.mult_add(xh, yh)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    ms, e2e_s = max_over_ranks([ms, e2e_s], world, device=f"cuda:{local}")
    solve = None
    if (args.solve or world == 1) and not args.no_solve:
        qed.set_global_parameter("GF_method", "L")
        qed.load_problem(prob, label + 100, model_name="bench_sq4x4", fmt="F")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, sec = qed.ground_state_solve(label + 100)
        t1 = time.perf_counter()
        qed.Green_function_solve(label + 100)
        G = qed.Green_function(W.matsubara(256), label=label + 100)
        t2 = time.perf_counter()
        solve = {"ground_state_seconds": t1 - t0, "E0": e, "sector": sec,
                 "green_function_seconds": t2 - t1, "G_iw0_00": [G[0, 0, 0].real, G[0, 0, 0].imag],
                 "what": "4x4 ground state (Lanczos) + band-Lanczos (p=16) Green function on 256 Matsubara "
                         "frequencies, beta=50"}
        fx = os.path.join(ROOT, "tests", "golden", "sq4x4_gs.json")
        if os.path.exists(fx):  # the reference's own ground state of this sector
            with open(fx) as f:
                r = json.load(f)
            solve["reference_ground_state"] = {"E0": r["E0"], "seconds": r["seconds"], "threads": r["threads"],
                                               "where": "one core of the build host (fixture tests/golden/sq4x4_gs.json)"}
            solve["E0_rel_diff"] = abs(e - r["E0"]) / abs(r["E0"])
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            Hr = cpu_baseline_sample()
            t0 = time.perf_counter()
            Hr.bench(1)
            dt = time.perf_counter() - t0
            del Hr  # released before the VCA line resets the oracle's model registry
            cpu = {"value": 16.0 * D / dt / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "one full H.v application of the 4x4 sector by the reference's "
                             "Hamiltonian_Factorized::mult_add (no threading in the reference's H.v)"}
    if rank != 0:
        return
    alg = 16.0 * D
    peak, src = peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    traffic = ncu_traffic(D)
    line = {
        "metric": METRIC, "value": aggregate_value(alg, ms, world), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "inputs": "larger than L2 (1.33 GB vectors), no flush",
                   "parallelism": f"replicas x{world}", "bytes_per_step": alg},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": src,
                     "unit_of_work": "one H.v (column pass k_hv_cols16w + row pass k_hv_rows16), 16 B per basis state"},
        "e2e": {"value": aggregate_value(alg, e2e_s * 1e3, world), "unit": UNIT, "h2d_bytes_per_step": 8 * D,
                "d2h_bytes_per_step": 8 * D,
                "path": "qed_hamiltonian_mult_add (y += H x) on pinned host buffers: x up in row blocks "
                        "overlapped with the row pass, the down-spin pass by row blocks with H x down overlapped "
                        "with it, y += H x on host threads; bound by the two transfers (H x needs all of x), "
                        "8 B per state each way"},
        "gpu_launches": 2 * args.steps,
        "hv_tuning": qed.hv_tuning_report(),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if solve:
        line["solve"] = solve
    if world == 1 and not args.no_secondary:
        line["secondary"] = secondary_lines("ours")
        line.update(secondary_summary(line["secondary"]))
    print(json.dumps(line), flush=True)


def batch_problems(args, rank=0, world=1):
    """The instances of one step, sharded round-robin over ranks (replicas)."""
    from pyqcm_b200 import workloads as W
    if args.workload == "batch":
        probs = W.random_batch(args.batch, seed=12345)
    else:
        probs = W.random_baths(args.batch, seed=4242)
    return probs[rank::world]


def _ref_solve_one(payload):
    """One instance through the reference (a worker process of the CPU pool)."""
    prob, label, method = payload
    from oracle import ref
    ref.set_param("GF_method", method)
    ref.load_problem(prob, label, model_name=f"refpool_{label}", fmt="F")
    e, _ = ref.ground_state(label)
    ref.green_solve(label)
    return e


BATCH_WORKLOADS = {
    "batch": "independent Hubbard clusters (2x2, 2x3, 2x4, chain 8, chain 10; U~U[0,12], mu~U[0,U], "
             "Neel field M~U[0,0.3]; every (N_up,N_dn) sector), ground state + band-Lanczos Green function",
    "baths": "2x2 plaquette + 8 bath orbitals, U=8, R0:N12:S0 (dim 853776), random baths; ground state + "
             "4x4 band-Lanczos Green function",
}


def batch_line(workload, batch, threads, steps, warmup, impl, world=1, rank=0, local=0, gpus=1):
    """ED solves/s on one of the batched workloads; returns the JSON dict (None on ranks > 0)."""
    metric = "ED solves/s"
    wl = BATCH_WORKLOADS[workload]
    ns = argparse.Namespace(workload=workload, batch=batch)
    probs = batch_problems(ns, rank, world)
    if impl == "reference":
        if rank != 0:
            return None
        import multiprocessing as mp
        cores = os.cpu_count() or 8
        n = min(len(probs), cores)
        sample = probs[:n]
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(cores) as pool:
            pool.map(_ref_solve_one, [(p, 9100 + i, "L") for i, p in enumerate(sample)], chunksize=1)
        dt = time.perf_counter() - t0
        v = n / dt
        return {"metric": metric, "value": v, "unit": "solves/s", "n_gpus": gpus, "steps": 1, "warmup": 0,
                "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": wl, "instances_per_step": n},
                "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                                 "sample": f"the first {n} instances, one process per core (the reference's ED "
                                           "is single-threaded per instance)"},
                "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    import torch
    import pyqcm_b200 as qed
    torch.cuda.set_device(local)
    qed.init(local)
    qed.set_global_parameter("GF_method", "L")

    def one_step(base):
        labels = []
        for i, p in enumerate(probs):
            qed.load_problem(p, base + i, model_name=f"bw_{p.name}_{base + i}", fmt="F")
            labels.append(base + i)
        t0 = time.perf_counter()
        qed.ground_state_solve_batch(labels, threads=threads)
        qed.Green_function_solve_batch(labels, threads=threads)
        G = [qed.Green_function(1j * np.pi / 50, label=l) for l in labels]  # results back on the host
        dt = time.perf_counter() - t0
        for l in labels:
            qed.erase_model_instance(l)
        return dt, G

    if warmup > 0:  # the code paths and allocations of every geometry, on a smaller batch
        full = probs
        probs = full[:min(len(full), 64)]
        one_step(200000)
        probs = full
    steps = max(1, min(steps, 3))
    busy = UtilSampler(local)
    busy.start()
    times = [one_step(300000 + 10000 * k)[0] for k in range(steps)]
    gpu_busy = busy.stop()
    dt = sum(times) / steps
    dt = max_over_ranks([dt], world, device=f"cuda:{local}")[0]
    if rank != 0:
        return None
    return {"metric": metric, "value": batch / dt, "unit": "solves/s", "n_gpus": world, "steps": steps,
            "warmup": min(warmup, 1), "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": wl, "instances_per_step": batch,
                                            "host_threads": threads or os.cpu_count()},
            "gpu_busy": gpu_busy,
            "e2e": {"value": batch / dt, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 16 * batch,
                    "path": "qed_ground_state_solve_batch + qed_Green_function_solve_batch + G(z) read back"}}


SECONDARY = (("batch", 1024), ("baths", 256))  # the stated sizes: 1024 random clusters, 256 bath points
VCA_SECONDARY_POINTS = 4096


def secondary_lines(impl):
    """The batched-solve metrics (and, for this solver, the VCA line) reported
    beside the H.v line of the default run."""
    out = []
    for wl, n in SECONDARY:
        line = batch_line(wl, n, 0, 1, 1, impl)
        if line:
            out.append(line)
    if impl == "ours":
        out.append(vca_line(VCA_SECONDARY_POINTS, 400, 0))
        out.append(cdmft_line())
    return out


def secondary_summary(lines):
    """Headline figures of the batched and VCA lines, as top-level keys."""
    out = {}
    for ln in lines:
        wl = ln.get("config", {}).get("workload", "")
        if ln.get("metric") == "ED solves/s":
            key = "batched_random_clusters" if wl == BATCH_WORKLOADS["batch"] else "batched_bath_points"
            out[key] = {"solves_per_s": ln["value"], "instances": ln["config"].get("instances_per_step"),
                        "gpu_busy_pct": (ln.get("gpu_busy") or {}).get("mean_pct"),
                        "cpu_pool": ln.get("cpu_baseline")}
        elif ln.get("metric", "").startswith("VCA"):
            out["vca"] = {k: ln.get(k) for k in ("value", "ed_only_seconds", "speedup", "surrogate_total_seconds",
                                                  "speedup_including_training", "breakeven_searches",
                                                  "max_omega_abs_diff", "max_grad_norm")}
            out["vca"]["training_points"] = ln["config"]["training_points"]
        elif ln.get("metric", "").startswith("CDMFT"):
            out["cdmft_bath_surrogate"] = {k: ln.get(k) for k in ("value", "plain_solves", "plain_seconds",
                                                                  "speedup", "surrogate_total_seconds",
                                                                  "breakeven_runs", "max_gamma_abs_diff")}
    return out


def run_batch_workload(args, world, rank, local):
    line = batch_line(args.workload, args.batch, args.threads, args.steps, args.warmup, args.impl,
                      world, rank, local, args.gpus)
    if line:
        print(json.dumps(line), flush=True)


VCA_WORKLOAD = ("VCA on the square lattice (t=1) tiled by 2x5 clusters (superlattice (2,0),(1,5)), "
                "half filling mu=U/2; variational Neel Weiss field M' and cluster chemical potential shift "
                "dmu; Omega from the ED ground state + band-Lanczos Green function (dim 63504) and a fixed "
                "grid of 64 Matsubara frequencies x 64x64 wavevectors; Newton-Raphson (3x3 central stencil, "
                "accuracy 2e-5) from (M', dmu) = (0.2, 0) with steps 0.02 (ED only) or from the surrogate's "
                "stationary point with steps 0.005 (surrogate-guided)")


VCA_REF_POINT = (7.0, 0.15, 0.0)  # (U, M', dmu) of the reference's timed Omega evaluation


def vca_reference_sample():
    """One Potthoff-functional evaluation of the 2x5 VCA workload by the reference's
    own lattice layer (the compiled oracle; ED ground state + Green function + the
    fixed grid) on one host core: (seconds, Omega)."""
    from oracle import ref
    from pyqcm_b200 import vca
    from pyqcm_b200 import workloads as W
    U, M, dmu = VCA_REF_POINT
    ref.set_param("GF_method", "L")
    ref.load_lattice(W.vca_2x5(U=U, M1=M, dmu=dmu), 0)
    w, p = W.regular_frequency_grid(2.0, 32, 32)
    ref.set_grids(w, p, (64, 64))
    t0 = time.perf_counter()
    om = ref.lattice_potthoff(0)
    return time.perf_counter() - t0, om


def vca_line(n_points, epochs, threads, Us=(5.0, 7.0, 9.0), local=0):
    """Surrogate-guided against ED-only VCA on the 2x5 cluster: training-data and
    training cost, then per U the wall time of both searches to the same stationary point."""
    import pyqcm_b200 as qed
    from pyqcm_b200 import lattice as LT, vca
    from pyqcm_b200 import workloads as W
    qed.init(local)
    qed.set_global_parameter("GF_method", "L")
    model = LT.LatticeModel(W.vca_2x5())
    w, p = W.regular_frequency_grid(2.0, 32, 32)
    ev = vca.OmegaEvaluator(model, [], w, p, (64, 64), to_values=vca.vca_values, threads=threads)
    box = [[4.0, 10.0], [0.0, 0.4], [-0.5, 0.5]]
    X = vca.training_points(n_points, box, seed=2024)
    t0 = time.perf_counter()
    y = np.concatenate([ev(X[i:i + 256]) for i in range(0, len(X), 256)])
    t_data = time.perf_counter() - t0
    sur = vca.SurrogateVCA(box, width=256, seed=0)
    t0 = time.perf_counter()
    losses = sur.fit(X, y, epochs=epochs, batch=256, lr=1e-3, seed=0)
    t_train = time.perf_counter() - t0
    acc = [2e-5, 2e-5]
    cert = 1e-6  # both searches end on |grad Omega| < 1e-6 from a 1e-4 central stencil
    runs = []
    for U in Us:
        f_ed = lambda P, U=U: ev(np.c_[np.full(len(P), U), P])
        n0 = ev.n_evals
        t0 = time.perf_counter()
        x_ed, _, g_ed, _, it_ed = vca.newton_raphson(f_ed, [0.2, 0.0], [0.02, 0.02], acc, certify=cert)
        t_ed = time.perf_counter() - t0
        n_ed = ev.n_evals - n0
        n0 = ev.n_evals
        t0 = time.perf_counter()
        x0 = sur.propose(U, [0.2, 0.0], [0.02, 0.02])
        x_s, _, g_s, _, it_s = vca.newton_raphson(f_ed, x0, [0.005, 0.005], acc, certify=cert)
        t_s = time.perf_counter() - t0
        n_s = ev.n_evals - n0
        x_poly = sur.propose(U, [0.2, 0.0], [0.02, 0.02], use_net=False)
        om = ev(np.c_[[U, U], np.vstack([x_ed, x_s])])
        runs.append({"U": U, "ed_only_s": t_ed, "surrogate_s": t_s, "ed_only_iterations": it_ed,
                     "surrogate_iterations": it_s, "ed_only_omega_evals": n_ed, "surrogate_omega_evals": n_s,
                     "x_ed_only": [float(v) for v in x_ed], "x_surrogate": [float(v) for v in x_s],
                     "grad_norm_ed_only": float(np.linalg.norm(g_ed)),
                     "grad_norm_surrogate": float(np.linalg.norm(g_s)),
                     "x_proposed": [float(v) for v in x0],
                     "x_proposed_polynomial_only": [float(v) for v in x_poly], "omega": float(om[0]),
                     "omega_abs_diff": float(abs(om[0] - om[1]))})
    t_sur = sum(r["surrogate_s"] for r in runs)
    t_ed = sum(r["ed_only_s"] for r in runs)
    om_here = float(ev(np.array([VCA_REF_POINT]))[0])
    t_ref, om_ref = vca_reference_sample()
    n_ed = sum(r["ed_only_omega_evals"] for r in runs)
    # what the surrogate costs in full, and after how many searches it pays for itself
    t_fixed = t_data + t_train
    gain = (t_ed - t_sur) / len(Us)
    breakeven = (t_fixed / gain) if gain > 0 else None
    return {"metric": "VCA wall time, surrogate-guided (same stationary point as ED-only within 1e-8)",
            "value": t_sur, "unit": "s", "n_gpus": 1, "steps": len(Us), "warmup": 0,
            "ms_per_step": 1e3 * t_sur / len(Us), "higher_is_better": False, "scaling": "replicas",
            "vs_baseline": None, "dtype": "f64 (ED, Omega); bf16 x bf16 -> f32 (surrogate)",
            "data": "synthetic", "config": {"workload": VCA_WORKLOAD, "U": list(Us),
                                            "training_points": n_points, "epochs": epochs,
                                            "stop": "certified |grad Omega| < 1e-6 (central stencil, step 1e-4)"},
            "ed_only_seconds": t_ed, "speedup": t_ed / t_sur if t_sur > 0 else None,
            "surrogate_total_seconds": t_fixed + t_sur,
            "surrogate_total_what": "training data (ED Omega at every training point) + training + the searches",
            "speedup_including_training": t_ed / (t_fixed + t_sur),
            "breakeven_searches": breakeven,
            "max_grad_norm": max(max(r["grad_norm_ed_only"], r["grad_norm_surrogate"]) for r in runs),
            "cpu_baseline": {"value": t_ref * n_ed, "unit": "s", "cores": 1, "kind": "reference",
                             "sample": f"one Potthoff-functional evaluation by the reference's compiled lattice "
                                       f"layer at (U, M', dmu) = {VCA_REF_POINT} took {t_ref:.2f} s on one host "
                                       f"core; value = that x the {n_ed} evaluations of the ED-only searches",
                             "omega_reference": om_ref, "omega_this_solver": om_here,
                             "omega_abs_diff": abs(om_ref - om_here)},
            "max_omega_abs_diff": max(r["omega_abs_diff"] for r in runs),
            "training": {"data_seconds": t_data, "omega_per_second": n_points / t_data,
                         "train_seconds": t_train, "first_loss": float(losses[0]), "last_loss": float(losses[-1])},
            "runs": runs}


CDMFT_WORKLOAD = ("CDMFT on the square lattice (t=1) tiled by 2x2 plaquettes with eight bath orbitals "
                  "(two per site; dim 924^2 = 853776 at half filling, mu=U/2), 16 bath parameters, "
                  "Legendre grid (1, 10, 5, 10, 5), host k-sum on 16x16 points, Broyden iterations, "
                  "least-squares bath fits with the exact Jacobian, converged when the bath moves less "
                  "than 1e-5 (per parameter, over two iterations)")


def cdmft_line(n_train=15, Us=(7.1, 7.7, 8.3, 8.9, 9.4), local=0):
    """Surrogate-proposed against model-bath starts of CDMFT on the bath-point cluster:
    training data (CDMFT converged by continuation in U), training, then per U the
    ED solves and wall time of both runs to the same hybridisation function."""
    import pyqcm_b200 as qed
    from pyqcm_b200 import cdmft, lattice as LT
    from pyqcm_b200 import workloads as W
    qed.init(local)
    qed.set_global_parameter("GF_method", "L")
    names = [f"eb{b}_1" for b in range(8)] + [f"tb{b}_1" for b in range(8)]
    rng = np.random.default_rng(7)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.3, 1, 8), U=8.0)
    model = LT.LatticeModel(prob)
    canon = lambda x: cdmft.canonical_bath(x, list(range(8)), list(range(8, 16)), [b // 2 for b in range(8)])
    args = dict(method="trf", accur=1e-5, maxiter=60, side=16)
    box = (6.5, 10.0)
    train_U = np.linspace(box[0], box[1], n_train)
    x0 = np.array([prob.params[n] for n in names])
    t0 = time.perf_counter()
    ok, baths, iters = cdmft.converge_baths(model, names, ["U"], train_U[:, None], x0, canonical=canon,
                                            label=910000, **args)
    t_data = time.perf_counter() - t0
    sur = cdmft.BathSurrogate(["U"], [box], names, seed=1)
    t0 = time.perf_counter()
    losses = sur.fit(train_U[ok, None], baths, epochs=800, seed=2)
    t_train = time.perf_counter() - t0
    runs = []
    for k, U in enumerate(Us):
        vals = dict(prob.params, U=U)
        t0 = time.perf_counter()
        plain = cdmft.CDMFT(model, names, values=vals, label=920000 + 100 * k, **args)
        t_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        start = sur.propose([U])
        guided = cdmft.CDMFT(model, names, values=vals, start=start, label=930000 + 100 * k, **args)
        t_guided = time.perf_counter() - t0
        bd = cdmft.BathDistance(model, names, vals)
        dg = float(np.max(np.abs(bd.gamma(plain.x, plain.grid.wr) - bd.gamma(guided.x, guided.grid.wr))))
        runs.append({"U": U, "plain_solves": plain.n_solves, "surrogate_solves": guided.n_solves,
                     "plain_s": t_plain, "surrogate_s": t_guided, "gamma_abs_diff": dg,
                     "E0_abs_diff": abs(plain.E0 - guided.E0),
                     "proposal_to_converged": float(np.max(np.abs(canon(guided.x) - start)))})
        plain.I.erase()
        guided.I.erase()
    t_p = sum(r["plain_s"] for r in runs)
    t_g = sum(r["surrogate_s"] for r in runs)
    gain = (t_p - t_g) / len(Us)
    return {"metric": "CDMFT wall time, surrogate-proposed starting bath (same hybridisation as the plain run)",
            "value": t_g, "unit": "s", "n_gpus": 1, "steps": len(Us), "warmup": 0,
            "ms_per_step": 1e3 * t_g / len(Us), "higher_is_better": False, "scaling": "replicas",
            "vs_baseline": None, "dtype": "f64 (ED, host, bath fits); bf16 x bf16 -> f32 (surrogate)",
            "data": "synthetic", "config": {"workload": CDMFT_WORKLOAD, "U": list(Us), "training_U": list(train_U),
                                            "model_bath_seed": 7},
            "plain_seconds": t_p, "speedup": t_p / t_g if t_g > 0 else None,
            "plain_solves": sum(r["plain_solves"] for r in runs),
            "surrogate_solves": sum(r["surrogate_solves"] for r in runs),
            "surrogate_total_seconds": t_data + t_train + t_g,
            "surrogate_total_what": "training data (CDMFT converged at every training U) + training + the runs",
            "breakeven_runs": (t_data + t_train) / gain if gain > 0 else None,
            "max_gamma_abs_diff": max(r["gamma_abs_diff"] for r in runs),
            "training": {"data_seconds": t_data, "points_converged": int(len(ok)), "iterations": iters.tolist(),
                         "train_seconds": t_train, "first_loss": float(losses[0]), "last_loss": float(losses[-1])},
            "runs": runs}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.workload == "vca":
            if rank == 0:
                print(json.dumps(vca_line(args.vca_points, args.vca_epochs, args.threads, local=local)), flush=True)
        elif args.workload == "cdmft":
            if rank == 0:
                print(json.dumps(cdmft_line(local=local)), flush=True)
        elif args.workload != "hv":
            run_batch_workload(args, world, rank, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
