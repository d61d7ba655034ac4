"""Benchmark of the ACO-for-CVRP hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one ACO epoch (construct all ants, iteration/global best, evaporate,
deposit) over the n=1000, K=8 workload: uniform integer coordinates in
[0,1000]^2 from seed 19001, depot (500,500), demands uniform in [1,100],
Q = ceil(sum(d)/(0.9 K)), 256 ants, 32-NN candidate lists.  The metric is
ant-steps/s (one ant-step = one customer move or depot return).

* value: device time of K epochs (CUDA events on the library's stream, the L2
  flushed by a 256 MiB write between epochs outside the events), all ranks'
  ant-steps over the max-over-ranks time.
* e2e: the same metric through the public C ABI with host buffers: per step
  one solve (upload of coordinates and demands, candidate lists, 64 epochs,
  download of the best routes and cost), timed on the host.
* roofline: the construct kernel (the dominant one), algorithmic bytes per
  ant-step k(4 + 4 + 1) (candidate id, weight, pheromone byte), over its mean
  event-timed duration.
* cpu_baseline / --impl reference: the reference's OpenMP solver
  (oracle/_ref/aco_vrp_omp.out, built from the reference sources) on the
  unit-demand twin of the workload with all host threads, fixed epochs; the
  oracle port (single thread) if that build is absent.

Multi-GPU (torchrun, one rank per GPU): every rank runs its own colony of 256
ants on the same instance with its own seed (weak scaling); the timed region
has no collective.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from vehicleroutingproblem_b200 import instances as I  # noqa: E402

WORKLOAD = dict(name="n1000 K8 uniform seed19001 demand[1,100] 256 ants 32-NN",
                ants=256, cand_k=32)
E2E_EPOCHS = 64
BYTES_PER_ANT_STEP = 32 * (4 + 4 + 1)
# dram__bytes_read.sum + dram__bytes_write.sum of one k_construct launch on
# this workload (profiles/k_construct_n1000.md): the candidate tables come
# from L2 into shared memory, so DRAM sees little of the algorithmic bytes.
CONSTRUCT_DRAM_BYTES_PER_LAUNCH = 234496
OMP_BIN = os.path.join(ROOT, "oracle", "_ref", "aco_vrp_omp.out")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# CPU baseline: the reference's OpenMP solver on the unit-demand twin
# ---------------------------------------------------------------------------

def _omp_run(vrp_path, K, ants, epochs, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), ACO_SOLVER_FIXED_EPOCHS=str(epochs),
               ACO_SOLVER_STAGNATION_EPOCHS="0", ACO_SOLVER_PROGRESS_INTERVAL_SECONDS="0")
    t0 = time.perf_counter()
    r = subprocess.run([OMP_BIN, vrp_path, str(K), str(ants), "1234"], env=env,
                       capture_output=True, text=True, timeout=600)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference OpenMP solver failed: {r.stderr[-400:]}")
    return dt


def cpu_baseline(inst, ants, target_s=12.0):
    """ant-steps/s of the reference's own CPU path, bounded sample."""
    n, K = inst.n, inst.vehicles
    steps_per_epoch = ants * (n + K)
    if os.path.exists(OMP_BIN):
        threads = os.cpu_count() or 1
        twin = inst.unit_twin()
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "twin.vrp")
            I.write_vrp(twin, path)
            t1 = _omp_run(path, K, ants, 2, threads)
            t2 = _omp_run(path, K, ants, 6, threads)
            per_epoch = max((t2 - t1) / 4.0, 1e-6)
            epochs = int(max(4, min(400, target_s / per_epoch)))
            ta = _omp_run(path, K, ants, 2, threads)
            tb = _omp_run(path, K, ants, 2 + epochs, threads)
            per_epoch = max((tb - ta) / epochs, 1e-9)
        return {"value": steps_per_epoch / per_epoch, "unit": "ant-steps/s", "cores": threads,
                "kind": "reference",
                "sample": (f"reference OpenMP solver (aco_parallel.c, no MPI) on the unit-demand "
                           f"twin, {ants} ants, {epochs} fixed epochs minus a 2-epoch run "
                           f"(set-up excluded), OMP_NUM_THREADS={threads}")}
    # Fallback: the oracle port, one thread, one epoch of `ants` ants.
    from oracle import oracle as O
    O.build()
    A, lut, thr = O.tables()
    k = WORKLOAD["cand_k"]
    cand = O.knn(inst.x, inst.y, k)
    lvl = O.levels(inst.x, inst.y, cand, k, thr)
    tau = np.full((n + 1) ** 2, O.params()["q_tau0"], np.uint8)
    w = O.weights(n, k, cand, lvl, tau, A, lut)
    t0 = time.perf_counter()
    steps = 0
    for a in range(ants):
        steps += O.construct_ant(inst.x, inst.y, inst.demand, K, inst.capacity, k, cand, w,
                                 1234, 0, a)[4]
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "ant-steps/s", "cores": 1, "kind": "port",
            "sample": f"oracle construct of {ants} ants, one epoch, one thread"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    inst = I.workload_n1000()
    cb = cpu_baseline(inst, WORKLOAD["ants"], target_s=max(4.0, 3.0 * args.steps))
    line = {"impl": "reference", "metric": "ant-steps/s", "value": cb["value"],
            "unit": "ant-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "n": inst.n, "K": inst.vehicles,
                       "ants": WORKLOAD["ants"], "cand_k": WORKLOAD["cand_k"],
                       "note": "reference CPU path runs the unit-demand twin (its parser "
                               "accepts demand 1 only)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "ant-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()

    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import torch
    import torch.distributed as dist
    from vehicleroutingproblem_b200 import _native

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    inst = I.workload_n1000()
    n, K, m, k = inst.n, inst.vehicles, WORKLOAD["ants"], WORKLOAD["cand_k"]
    # A dedicated stream (the default stream's handle is 0, which the C ABI
    # reads as "use your own stream"): the library's kernels, the L2 flush and
    # the timing events all go to it.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = _native.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.setup_instance(inst, ants=m, cand_k=k, seed=1234 + 7919 * rank)

    ctx.enqueue_epochs(args.warmup)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    steps0 = ctx.state().total_steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        wall0 = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(i & 0xff)
            evs[i][0].record(stream)
            ctx.enqueue_epochs(1)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    if world > 1:
        dist.barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    st = ctx.state()
    steps_done = st.total_steps - steps0
    assert st.error == 0 and st.epochs == args.warmup + args.steps

    # Per-kernel device times (event between every kernel), for the roofline.
    kms = ctx.profile_epochs(32) / 32.0
    t = torch.tensor([dev_ms, float(steps_done)], dtype=torch.float64, device="cuda")
    if world > 1:
        tmax = t.clone()
        dist.all_reduce(tmax[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tmax[1:2], op=dist.ReduceOp.SUM)
        t = tmax
    dev_ms_max, steps_all = float(t[0]), float(t[1])
    value = steps_all / (dev_ms_max / 1e3)

    # End to end through the public API with host buffers.
    e2e_vals = []
    h2d = (n + 1) * (8 + 4) + 4095 * 4 + 2 * 256 * 4
    d2h = (n + 2 * K) * 4 + K * 4
    for i in range(args.e2e_steps):
        t0 = time.perf_counter()
        with _native.Context(local) as c2:
            c2.setup_instance(inst, ants=m, cand_k=k, seed=99 + i, fixed_epochs=E2E_EPOCHS)
            s2 = c2.run(E2E_EPOCHS)
            c2.best()
        dt = time.perf_counter() - t0
        if i > 0:  # first call pays the one-time module load
            e2e_vals.append(s2.total_steps / dt)
    e2e = statistics.median(e2e_vals) if e2e_vals else None
    if world > 1:
        te = torch.tensor([e2e or 0.0], dtype=torch.float64, device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.SUM)
        e2e = float(te[0])

    peak, peak_kind = load_peaks()
    construct_s = float(kms[1]) / 1e3
    steps_per_launch = steps_done / args.steps
    achieved = BYTES_PER_ANT_STEP * steps_per_launch / construct_s / 1e9
    total_k = float(kms.sum())
    clocks = clk.summary()

    if rank == 0:
        line = {
            "metric": "ant-steps/s", "value": value, "unit": "ant-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "int32 weights + u8 pheromone (f64 route costs)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "n": n, "K": K, "capacity": inst.capacity,
                       "ants": m, "cand_k": k, "step": "one epoch",
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "parallelism": f"{world} independent colonies" if world > 1 else "1 GPU"},
            "wall_s": wall,
            "gpu_launches": 4 * args.steps,
            "kernels_us": {"weights": float(kms[0]) * 1e3, "construct": float(kms[1]) * 1e3,
                           "best": float(kms[2]) * 1e3, "evap_deposit": float(kms[3]) * 1e3},
            "kernel_share": {"construct": float(kms[1]) / total_k if total_k else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": CONSTRUCT_DRAM_BYTES_PER_LAUNCH,
                         "kernel": "k_construct", "peak_kind": peak_kind,
                         "bytes_per_ant_step": BYTES_PER_ANT_STEP},
            "e2e": {"value": e2e, "unit": "ant-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "step": f"one solve through the C ABI: upload, candidates, {E2E_EPOCHS} "
                            "epochs, download of the best routes"},
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(inst, m)
            except Exception as exc:  # reported, not fatal
                line["cpu_baseline"] = {"error": str(exc)[:200]}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
