"""Benchmark of the ACO-for-CVRP hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload n1000|small|clustered2000|large16000|large32000|
                                batched|learned|costdist]

Default workload (n1000): n=1000, K=8 uniform integer coordinates in
[0,1000]^2 from seed 19001, depot (500,500), demands uniform in [1,100],
Q = ceil(sum(d)/(0.9 K)), 256 ants, 32-NN candidate lists.  A step is one
ACO epoch (construct all ants, iteration/global best, evaporate, deposit);
the metric is ant-steps/s (one ant-step = one customer move or depot return).
small: n=100, K=4, demands [1,30], seed 1001, 128 ants, 20-NN.
clustered2000: n=2000, K=16, 70% in 8 Gaussian clusters, 1024 ants, 32-NN.
large16000 / large32000: n=16000, K=16 / n=32000, K=32, uniform, 256 ants,
32-NN (pheromone matrices of 256 MB / 1 GB, beyond L2).
batched: 512 instances (n~U[50,500], K=ceil(n/60), seeds 30000-30511), 64
ants, 300 epochs each, all in one persistent launch; the autotuner chooses
the candidate-list length (16, 20 or 32: the fastest within 0.5 % of the
best mean final cost) and the launch shape; a step is one solve of the
whole batch and the metric is instances/s.
learned: the learned prior's time-to-cost against plain eta on 256 held-out
n=1000 instances (training set, training and evaluation inside the run).
costdist: not a throughput line -- the best cost over seeds at fixed epochs
of this library's CLI (both depot rules) and the reference's own CUDA
solver, same CLI contract, same GPU, unit-demand twin of n1000.

* value: device time (CUDA events on the library's stream), L2 flushed by a
  256 MiB write between steps outside the events, all ranks' work over the
  max-over-ranks time.
* e2e: the same metric through the public C ABI with host buffers (per step
  one solve: upload, candidate lists, epochs, download of the result), timed
  on the host.
* roofline: the dominant kernel, algorithmic bytes per ant-step k(4 + 4 + 1)
  (candidate id, weight, pheromone byte) over its mean event-timed duration.
* roofline_update: the pheromone evaporation sweep, 2 (n+1)^2 bytes per
  launch over its mean event-timed duration, timed alone; where the
  workload's matrices fit in L2 (n1000, small, clustered2000) the line also
  carries roofline_update_hbm, the same sweep on an n=16000 matrix pair, and
  roofline_seq_update_hbm, the sequential path's FP64 update on an n=16000
  matrix (16 bytes per cell).
* batched / learned_time_to_cost (default n1000 run only, --no-extras skips
  them): the other two figures of the headline metric -- instances/s of the
  batched form on the full 512-instance batch beside the single-instance
  solver looped over a sample, and the learned prior's time-to-cost against
  plain eta (and a tuned-beta control) with 512 training and 8 held-out
  instances; other_configs: the small and clustered2000 workloads over 50
  epochs each beside the reference's OpenMP solver.
* cli_same_contract / reference_cuda_same_gpu (reference arm): this
  library's aco_vrp_cuda.out and the reference's own CUDA solver (built from
  its sources for sm_100a) run through the same CLI on the same GPU and the
  unit-demand twin, epochs per second from their final progress line under
  ACO_SOLVER_TIMEOUT_SECONDS.
* cpu_baseline / --impl reference: the reference's OpenMP solver
  (oracle/_ref/aco_vrp_omp.out, built from the reference sources) on the
  unit-demand twins with all host threads and fixed epochs; the oracle port
  (single thread) if that build is absent.

Multi-GPU (torchrun, one rank per GPU).  Single-instance workloads split
one colony over the ranks (vehicleroutingproblem_b200.sharding): every rank
builds its own m ants on a replicated pheromone matrix, and each epoch ends
with one NCCL all-gather of the ranks' best-ant packets, after which every
rank applies the same deposits -- N ranks run one colony of N m ants (weak
scaling: the ants per GPU stay fixed).  `--colony sharded` takes that path on
one GPU as well.  The batched workload splits the instances over the ranks
with no collective in the timed region (strong scaling).
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

WORKLOADS = {
    "n1000": dict(factory=I.workload_n1000, ants=256, cand_k=32, e2e_epochs=64,
                  name="n1000 K8 uniform seed19001 demand[1,100] 256 ants 32-NN"),
    "small": dict(factory=I.workload_small, ants=128, cand_k=20, e2e_epochs=200,
                  name="n100 K4 uniform seed1001 demand[1,30] 128 ants 20-NN"),
    "clustered2000": dict(factory=I.workload_clustered2000, ants=1024, cand_k=32, e2e_epochs=32,
                          name="n2000 K16 clustered seed29001 demand[1,100] 1024 ants 32-NN"),
    "large16000": dict(factory=lambda: I.workload_large(16000), ants=256, cand_k=32, e2e_epochs=8,
                       name="n16000 K16 uniform seed160001 demand[1,100] 256 ants 32-NN"),
    "large32000": dict(factory=lambda: I.workload_large(32000), ants=256, cand_k=32, e2e_epochs=4,
                       name="n32000 K32 uniform seed320001 demand[1,100] 256 ants 32-NN"),
}
# L2 of one B200 (bytes): a pheromone matrix pair below it stays L2-resident
# between sweeps.
L2_BYTES = 126 * 1024 * 1024
BATCHED = dict(count=512, seed0=30000, ants=64, cand_k=16, epochs=300,
               name="512 instances n~U[50,500] K=ceil(n/60) seeds 30000-30511 demand[1,100] "
                    "64 ants, candidate lists of 16/20/32 chosen by the autotuner, 300 epochs")
# dram__bytes_read.sum + dram__bytes_write.sum of one k_construct launch on
# the n1000 workload, from an ncu capture made separately (not measured in
# this run): the candidate tables come from L2 into shared memory, so DRAM
# sees little of the algorithmic bytes.  Other workloads report null.
CONSTRUCT_DRAM_BYTES_PER_LAUNCH = {"n1000": 243456}
# The same for one k_evaporate_to launch, keyed by n (ncu capture made
# separately, mean of two launches on the large16000 workload): reads are the
# 256 MB source matrix, writes fall short of 256 MB by what is still in L2
# when the launch ends.
UPDATE_DRAM_BYTES_PER_LAUNCH = {16000: 460186752}
OMP_BIN = os.path.join(ROOT, "oracle", "_ref", "aco_vrp_omp.out")
REF_CUDA_BIN = os.path.join(ROOT, "oracle", "_ref", "aco_vrp_cuda_ref.out")
SEQ_BIN = os.path.join(ROOT, "oracle", "_ref", "aco_vrp_seq.out")
OUR_CLI = os.path.join(ROOT, "aco_vrp_cuda.out")
CLI_SECONDS = 4.0


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
            time.sleep(0.5)  # let the sampler start before the timed region
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
# CPU baseline: the reference's OpenMP solver on unit-demand twins
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


def _omp_epoch_seconds(inst, ants, threads, target_s, td):
    """Seconds per epoch of the reference OpenMP solver, set-up excluded."""
    path = os.path.join(td, inst.name + ".vrp")
    I.write_vrp(inst.unit_twin(), path)
    t1 = _omp_run(path, inst.vehicles, ants, 2, threads)
    t2 = _omp_run(path, inst.vehicles, ants, 6, threads)
    per = max((t2 - t1) / 4.0, 1e-6)
    epochs = int(max(4, min(400, target_s / per)))
    ta = _omp_run(path, inst.vehicles, ants, 2, threads)
    tb = _omp_run(path, inst.vehicles, ants, 2 + epochs, threads)
    return max((tb - ta) / epochs, 1e-9), epochs


def omp_candidate_k(n):
    """Candidate-list length the reference OpenMP solver picks for n on this
    host: 0.7 L3 / ((n+1) 8 B), clamped to [16, 512], 32 when the L3 size is
    unknown (tune_candidate_k and get_l3_cache_size,
    src/openmp-mpi/aco_parallel.c:143-174)."""
    l3 = 0
    try:
        with open("/sys/devices/system/cpu/cpu0/cache/index3/size") as f:
            txt = f.read().strip()
        num = int("".join(ch for ch in txt if ch.isdigit()) or 0)
        unit = next((ch for ch in txt if ch in "KMGTkmgt"), "")
        l3 = num * {"k": 1 << 10, "m": 1 << 20, "g": 1 << 30}.get(unit.lower(), 1)
    except OSError:
        pass
    if l3 <= 0:
        return {"k": 32, "effective_k": min(32, n), "l3_bytes": None}
    k = max(16, min(512, int(l3 * 0.7 / ((n + 1) * 8.0))))
    # slots past the n customers stay empty
    return {"k": k, "effective_k": min(k, n), "l3_bytes": l3}


def cpu_baseline_seq_construct(inst, cand_k, target_s=10.0):
    """ant-steps/s of the reference's own sequential construction
    (build_ant_solution, src/seq/aco_sequential.c:616-681, compiled from its
    sources into oracle/_ref/libseqref.so) on the unit-demand twin, fed this
    path's candidate lists and weights at the initial pheromone and recorded
    draws.  For large n, where the reference solvers' own set-up (an
    O(n^2 k) candidate build over a candidate list of up to 512) does not
    finish in a bounded sample.  The distance matrix the harness builds per
    call is excluded by timing 1 and 1 + a ants."""
    from oracle import oracle as O
    O.build()
    twin = inst.unit_twin()
    n, K = twin.n, twin.vehicles
    A, lut, thr = O.tables()
    cand = O.knn(twin.x, twin.y, cand_k)
    lvl = O.levels(twin.x, twin.y, cand, cand_k, thr)
    tau = np.full((n + 1) ** 2, O.params()["q_tau0"], np.uint8)
    w = O.weights(n, cand_k, cand, lvl, tau, A, lut)
    rs = np.random.RandomState(7)

    def run(m):
        dr = rs.randint(0, 1 << 24, size=(m, n + K + 8)).astype(np.uint32)
        t0 = time.perf_counter()
        res = O.ref_construct_ants(twin.x, twin.y, K, twin.capacity, cand_k, cand, w, dr)
        return time.perf_counter() - t0, sum(int(r[1].sum()) - K for r in res)

    t1, s1 = run(1)
    extra = 2
    while True:
        t2, s2 = run(1 + extra)
        if t2 - t1 > target_s / 4 or extra >= 64:
            break
        extra *= 2
    per_step = max(t2 - t1, 1e-9) / max(s2 - s1, 1)
    return {"value": 1.0 / per_step, "unit": "ant-steps/s", "cores": 1, "kind": "reference",
            "sample": (f"the reference's sequential build_ant_solution (compiled from its "
                       f"sources) on the unit-demand twin, {extra} ants with recorded draws on "
                       f"this path's {cand_k}-NN lists and initial weights, one thread; the "
                       "reference solvers' own set-up is O(n^2 k) and does not finish in a "
                       "bounded sample at this n")}


def cpu_baseline(inst, ants, target_s=12.0, cand_k=32):
    """ant-steps/s of the reference's own CPU path, bounded sample."""
    n, K = inst.n, inst.vehicles
    if n > 4000:
        from oracle import oracle as O
        if O.ref_available():
            return cpu_baseline_seq_construct(inst, cand_k)
    if os.path.exists(OMP_BIN):
        threads = os.cpu_count() or 1
        steps_per_epoch = ants * (n + K)
        with tempfile.TemporaryDirectory() as td:
            per_epoch, epochs = _omp_epoch_seconds(inst, ants, threads, target_s, td)
        kc = omp_candidate_k(n)
        return {"value": steps_per_epoch / per_epoch, "unit": "ant-steps/s", "cores": threads,
                "kind": "reference", "candidate_k": kc,
                "sample": (f"reference OpenMP solver (aco_parallel.c, no MPI) on the unit-demand "
                           f"twin, {ants} ants, {epochs} fixed epochs minus a 2-epoch run "
                           f"(set-up excluded), OMP_NUM_THREADS={threads}, its own L3-tuned "
                           f"candidate list of {kc['k']} (this GPU path uses {cand_k})")}
    steps_per_epoch = ants * (n + K)
    # Fallback: the oracle port, one thread, one epoch of `ants` ants.
    from oracle import oracle as O
    O.build()
    A, lut, thr = O.tables()
    cand = O.knn(inst.x, inst.y, cand_k)
    lvl = O.levels(inst.x, inst.y, cand, cand_k, thr)
    tau = np.full((n + 1) ** 2, O.params()["q_tau0"], np.uint8)
    w = O.weights(n, cand_k, cand, lvl, tau, A, lut)
    t0 = time.perf_counter()
    steps = 0
    for a in range(ants):
        steps += O.construct_ant(inst.x, inst.y, inst.demand, K, inst.capacity, cand_k, cand,
                                 w, 1234, 0, a)[4]
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "ant-steps/s", "cores": 1, "kind": "port",
            "sample": f"oracle construct of {ants} ants, one epoch, one thread"}


def cpu_baseline_batched(insts, target_s=15.0):
    """instances/s of the reference OpenMP solver over a sample of the batch
    (each instance: its own process, 64 ants, 300 fixed epochs), scaled to the
    whole batch by work (n + K)."""
    if not os.path.exists(OMP_BIN):
        return {"error": "oracle/_ref not built"}
    threads = os.cpu_count() or 1
    spent, idx = 0.0, []
    with tempfile.TemporaryDirectory() as td:
        for i in range(0, len(insts), max(1, len(insts) // 32)):
            per_epoch, _ = _omp_epoch_seconds(insts[i], BATCHED["ants"], threads, 0.5, td)
            spent += per_epoch * BATCHED["epochs"]
            idx.append(i)
            if spent > target_s:
                break
    w = np.array([x.n + x.vehicles for x in insts], float)
    total = spent * w.sum() / w[idx].sum()
    return {"value": len(insts) / total, "unit": "instances/s", "cores": threads,
            "kind": "reference",
            "sample": (f"reference OpenMP solver on the unit-demand twins of {len(idx)} of the "
                       f"{len(insts)} instances, 64 ants, per-epoch time x 300 epochs, scaled "
                       f"to the batch by n+K, OMP_NUM_THREADS={threads}")}


def cli_epoch_rate(binary, inst, ants, seconds=CLI_SECONDS, extra_env=None):
    """Epoch rate of a solver binary with the reference CLI contract
    (`<vrp> <K> <m> <seed>`, ACO_SOLVER_* env) on the unit-demand twin, from
    its last `[progress][cuda] epoca=E | ... tempo_trascorso=S s` line under
    ACO_SOLVER_TIMEOUT_SECONDS (the timer starts after set-up)."""
    import re
    twin = inst.unit_twin()
    n, K = twin.n, twin.vehicles
    env = dict(os.environ, ACO_SOLVER_TIMEOUT_SECONDS=str(seconds),
               ACO_SOLVER_STAGNATION_EPOCHS="0", ACO_SOLVER_PROGRESS_INTERVAL_SECONDS="0")
    env.pop("ACO_SOLVER_FIXED_EPOCHS", None)
    env.update(extra_env or {})
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, twin.name + ".vrp")
        I.write_vrp(twin, path)
        r = subprocess.run([binary, path, str(K), str(ants), "1234"], env=env,
                           capture_output=True, text=True, timeout=seconds + 300)
    if r.returncode != 0:
        return {"error": f"exit {r.returncode}: {r.stderr[-300:]}"}
    prog = re.findall(r"epoca=(\d+) .*tempo_trascorso=([0-9.]+)s", r.stdout)
    cost = re.findall(r"best cost: ([0-9.]+)", r.stdout)
    if not prog:
        return {"error": "no progress line"}
    e, sec = int(prog[-1][0]), float(prog[-1][1])
    return {"epochs": e, "seconds": sec, "epochs_per_s": e / sec,
            "ant_steps_per_s_max": ants * (n + K) * e / sec,
            "best_cost": float(cost[-1]) if cost else None,
            "instance": f"unit-demand twin n={n} K={K} capacity={twin.capacity}",
            "ants": ants, "timeout_s": seconds}


def cli_trajectory(binary, twin, ants, seed, seconds, extra_env=None):
    """Every progress line of one solver binary run with the reference CLI
    contract on a unit-demand instance: [(epoch, elapsed s, best cost)]."""
    import re
    env = dict(os.environ, ACO_SOLVER_TIMEOUT_SECONDS=str(seconds),
               ACO_SOLVER_STAGNATION_EPOCHS="0", ACO_SOLVER_PROGRESS_INTERVAL_SECONDS="0")
    env.pop("ACO_SOLVER_FIXED_EPOCHS", None)
    env.update(extra_env or {})
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, twin.name + ".vrp")
        I.write_vrp(twin, path)
        r = subprocess.run([binary, path, str(twin.vehicles), str(ants), str(seed)], env=env,
                           capture_output=True, text=True, timeout=seconds + 300)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} exit {r.returncode}: {r.stderr[-300:]}")
    return [(int(e), float(t), float(c)) for e, t, c in re.findall(
        r"epoca=(\d+) .*tempo_trascorso=([0-9.]+)s .*best_cost=([0-9.]+)", r.stdout)]


def run_costdist(args):
    """Cost-quality distribution over seeds of three solvers behind the same
    CLI on the same GPU: this library's aco_vrp_cuda.out with the default
    (sequential) rules and with ACO_CUDA_DEPOT_RULE=cuda_ref, and the
    reference's own CUDA solver built from its sources for sm_100a
    (src/cuda/aco_cuda.cu, aco_cuda_kernels.cu), on the unit-demand twin of
    the n1000 workload.  Each run has the same wall-time limit; the best
    cost is read at fixed epochs from the progress lines (printed at epoch
    1, every 10th epoch and on each improvement)."""
    twin = I.workload_n1000().unit_twin()
    ants, secs = 256, args.costdist_seconds
    marks = (10, 100, 300, 1000)
    solvers = [("b200 default rule", OUR_CLI, {}),
               ("b200 cuda_ref rule", OUR_CLI, {"ACO_CUDA_DEPOT_RULE": "cuda_ref"}),
               ("reference CUDA solver", REF_CUDA_BIN, {})]
    out = {}
    for name, binary, env in solvers:
        if not os.path.exists(binary):
            out[name] = {"error": f"{binary} not built"}
            continue
        per_seed = []
        for seed in range(1, args.costdist_seeds + 1):
            tr = cli_trajectory(binary, twin, ants, seed, secs, env)
            at = {}
            for mk in marks:
                seen = [c for e, _, c in tr if e <= mk]
                at[mk] = seen[-1] if seen and tr[-1][0] >= mk else None
            e_last, t_last, c_last = tr[-1]
            per_seed.append({"seed": seed, "best_at": at, "final": c_last, "epochs": e_last,
                             "epochs_per_s": e_last / t_last if t_last > 0 else None})

        def stats(v):
            v = np.array([x for x in v if x is not None], float)
            if not len(v):
                return None
            return {"mean": float(v.mean()), "median": float(np.median(v)),
                    "std": float(v.std(ddof=1)) if len(v) > 1 else 0.0,
                    "min": float(v.min()), "max": float(v.max()), "runs": int(len(v))}
        out[name] = {"best_at_epoch": {str(mk): stats([r["best_at"][mk] for r in per_seed])
                                       for mk in marks},
                     "final": stats([r["final"] for r in per_seed]),
                     "epochs_per_s": stats([r["epochs_per_s"] for r in per_seed]),
                     "per_seed": per_seed}
    line = {"metric": "best cost over seeds at fixed epochs (same CLI, same GPU)",
            "unit": "route cost (FP64)", "higher_is_better": False,
            "config": {"instance": f"unit-demand twin of the n1000 workload: n={twin.n} "
                                   f"K={twin.vehicles} capacity={twin.capacity}",
                       "ants": ants, "seeds": args.costdist_seeds, "timeout_s": secs,
                       "stagnation": "off"},
            "solvers": out}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    if args.workload == "batched":
        insts = I.batched_instances(BATCHED["count"], BATCHED["seed0"])
        cb = cpu_baseline_batched(insts)
        cfg = {"workload": BATCHED["name"], "instances": BATCHED["count"]}
        metric, unit = "instances/s", "instances/s"
    else:
        wl = WORKLOADS[args.workload]
        inst = wl["factory"]()
        cb = cpu_baseline(inst, wl["ants"], target_s=max(4.0, min(20.0, 0.01 * args.steps)),
                          cand_k=wl["cand_k"])
        cfg = {"workload": wl["name"], "n": inst.n, "K": inst.vehicles, "ants": wl["ants"],
               "cand_k": wl["cand_k"]}
        metric, unit = "ant-steps/s", "ant-steps/s"
    cfg["note"] = "reference CPU path runs the unit-demand twins (its parser accepts demand 1 only)"
    ref_gpu = None
    if args.workload != "batched" and os.path.exists(REF_CUDA_BIN):
        # The reference's own CUDA solver (built from its sources for sm_100a)
        # on this machine's GPU, same CLI contract: the GPU bar to beat.
        try:
            ref_gpu = cli_epoch_rate(REF_CUDA_BIN, inst, wl["ants"])
        except Exception as exc:  # reported, not fatal
            ref_gpu = {"error": str(exc)[:200]}
    line = {"impl": "reference", "metric": metric, "value": cb.get("value"), "unit": unit,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic", "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": cb.get("value"), "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if ref_gpu is not None:
        line["reference_cuda_same_gpu"] = ref_gpu
    if args.workload != "batched" and inst.n <= 4000 and os.path.exists(SEQ_BIN):
        # The reference's sequential solver on one host core, same CLI.
        try:
            line["reference_seq_1core"] = cli_epoch_rate(SEQ_BIN, inst, wl["ants"], seconds=10.0)
        except Exception as exc:  # reported, not fatal
            line["reference_seq_1core"] = {"error": str(exc)[:200]}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def update_roofline(ctx, n, launches, peak, peak_kind):
    """Roofline of the pheromone evaporation sweep (k_evaporate_to, the
    reference's kernel_evaporate_tau) on this context's matrix: 2 (n+1)^2
    algorithmic bytes (each byte read once and written once) per launch over
    the device time of one launch, the sweep timed alone: `launches`
    launches back to back between two CUDA events (after one untimed)."""
    ms = ctx.profile_update(launches)
    nbytes = 2 * (n + 1) ** 2
    achieved = nbytes / (ms / 1e3) / 1e9
    resident = nbytes <= L2_BYTES
    return {"bound": "hbm", "kernel": "k_evaporate_to", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "n": n,
            "bytes_per_launch": nbytes, "us_per_launch": ms * 1e3, "launches": launches,
            "timing": "launches back to back between two CUDA events on the sweep's stream",
            "residency": ("L2-resident: both matrices fit in L2, so this is not an HBM figure"
                          if resident else "HBM: the matrices exceed L2"),
            "traffic": UPDATE_DRAM_BYTES_PER_LAUNCH.get(n),
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                               "captured separately" if n in UPDATE_DRAM_BYTES_PER_LAUNCH
                               else None)}


def seq_update_roofline(torch, ctx, n, K, launches, peak, peak_kind):
    """Roofline of the sequential path's FP64 pheromone update
    (aco_b200_seq_pheromone_update; the reference's evaporation, deposits,
    MMAS clamp and reset loops, src/seq/aco_sequential.c:829-886) on an
    (n+1)^2 FP64 matrix: 16 algorithmic bytes per cell (each cell read and
    written once) over the mean CUDA-event time of one update, with the
    stagnation reset on; the solutions are two ants of `ctx` (set up on the
    same instance)."""
    from vehicleroutingproblem_b200 import _native
    L = _native.load()
    ctx.construct(0)
    nodes, lens, cost, _, _, _ = ctx.ants()
    sol = [(torch.from_numpy(nodes[a][: lens[a].sum()].astype(np.int32)).cuda(),
            torch.from_numpy(lens[a].astype(np.int32)).cuda(), float(cost[a])) for a in (0, 1)]
    tau = torch.full(((n + 1) * (n + 1),), 0.01, dtype=torch.float64, device="cuda")
    scratch = torch.zeros(L.aco_b200_seq_update_scratch_bytes(n), dtype=torch.uint8,
                          device="cuda")
    stream = torch.cuda.current_stream()
    tmax = 1.0 / (0.9 * sol[1][2])

    def call():
        return L.aco_b200_seq_pheromone_update(
            tau.data_ptr(), n, K, sol[0][0].data_ptr(), sol[0][1].data_ptr(), 0.3 / sol[0][2],
            sol[1][0].data_ptr(), sol[1][1].data_ptr(), 0.7 / sol[1][2], 0.1, 0.05 * tmax, tmax,
            1, 1.0, scratch.data_ptr(), stream.cuda_stream)

    assert call() == 0  # warm-up
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(launches)]
    for e0, e1 in evs:
        e0.record(stream)
        assert call() == 0
        e1.record(stream)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs) / launches
    nbytes = 16 * (n + 1) ** 2
    achieved = nbytes / (ms / 1e3) / 1e9
    del tau, scratch
    return {"bound": "hbm", "kernel": "k_seq_sweep + k_seq_mark + k_seq_deposit",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "n": n, "bytes_per_update": nbytes,
            "us_per_update": ms * 1e3, "launches": launches, "traffic": None,
            "note": ("FP64 matrix of the sequential path; the reference's loops make three "
                     "passes over it (48 bytes per cell with the reset), this update one")}


def timed_steps(torch, stream, steps, enqueue, flush):
    """Device ms of `steps` calls of enqueue(), each bracketed by events, the
    L2 flushed between steps outside the events."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for i in range(steps):
        flush.fill_(i & 0xff)
        evs[i][0].record(stream)
        enqueue()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


def run_single(args, rank, world, local, torch, dist, _native):
    wl = WORKLOADS[args.workload]
    inst = wl["factory"]()
    n, K, m, k = inst.n, inst.vehicles, wl["ants"], wl["cand_k"]
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
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        dev_ms = timed_steps(torch, stream, args.steps, lambda: ctx.enqueue_epochs(1), flush)
        wall = time.perf_counter() - wall0
    if world > 1:
        dist.barrier()
    st = ctx.state()
    steps_done = st.total_steps - steps0
    assert st.error == 0 and st.epochs == args.warmup + args.steps
    kms = ctx.profile_epochs(32) / 32.0
    peak, peak_kind = load_peaks()
    roof_upd = update_roofline(ctx, n, 200 if n <= 4000 else 50, peak, peak_kind)
    roof_upd_hbm = roof_seq_hbm = None
    if rank == 0 and (n + 1) ** 2 * 2 <= L2_BYTES and not args.no_large_update:
        # The matrix of this workload stays in L2; the same sweep on an
        # n=16000 matrix pair (512 MB) gives the HBM figure.
        with _native.Context(local) as cl:
            big = I.workload_large(16000)
            cl.set_stream(stream.cuda_stream)
            cl.setup_instance(big, ants=32, cand_k=k, seed=5)
            roof_upd_hbm = update_roofline(cl, big.n, 50, peak, peak_kind)
            roof_seq_hbm = seq_update_roofline(torch, cl, big.n, big.vehicles, 10, peak,
                                               peak_kind)
    t = torch.tensor([dev_ms, float(steps_done)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
    dev_ms_max, steps_all = float(t[0]), float(t[1])
    value = steps_all / (dev_ms_max / 1e3)

    e2e_vals = []
    h2d = (n + 1) * (8 + 4) + 4095 * 4 + 2 * 256 * 4
    d2h = (n + 2 * K) * 4 + K * 4
    # One context serves every solve (as a solver service would keep it):
    # each step uploads the instance from host memory, builds the candidate
    # lists, runs the epochs and downloads the best routes; the context's
    # device buffers and epoch graphs are reused across solves.
    c2 = _native.Context(local)
    for i in range(args.e2e_steps):
        t0 = time.perf_counter()
        c2.setup_instance(inst, ants=m, cand_k=k, seed=99 + i, fixed_epochs=wl["e2e_epochs"])
        s2 = c2.run(wl["e2e_epochs"])
        c2.best()
        dt = time.perf_counter() - t0
        if i > 0:  # the first call pays the one-time allocations and graph capture
            e2e_vals.append(s2.total_steps / dt)
    c2.close()
    e2e = statistics.median(e2e_vals) if e2e_vals else None
    if world > 1:
        te = torch.tensor([e2e or 0.0], dtype=torch.float64, device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.SUM)
        e2e = float(te[0])

    bytes_per_step = k * (4 + 4 + 1)
    achieved = bytes_per_step * (steps_done / args.steps) / (float(kms[1]) / 1e3) / 1e9
    total_k = float(kms.sum())
    line = None
    if rank == 0:
        line = {
            "metric": "ant-steps/s", "value": value, "unit": "ant-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "int32 weights + u8 pheromone (f64 route costs)",
            "data": "synthetic",
            "solutions_per_s": world * m * args.steps / (dev_ms_max / 1e3),
            "config": {"workload": wl["name"], "n": n, "K": K, "capacity": inst.capacity,
                       "ants": m, "cand_k": k, "step": "one epoch",
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "parallelism": f"{world} colonies, one per GPU" if world > 1 else "1 GPU"},
            "wall_s": wall,
            "gpu_launches": 4 * args.steps,
            "kernels_us": {"weights": float(kms[0]) * 1e3, "construct": float(kms[1]) * 1e3,
                           "evaporate (beside construct in the graph)": float(kms[2]) * 1e3,
                           "best_deposit": float(kms[3]) * 1e3},
            "kernel_share": {"construct": float(kms[1]) / total_k if total_k else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": CONSTRUCT_DRAM_BYTES_PER_LAUNCH.get(args.workload),
                         "kernel": "k_construct", "peak_kind": peak_kind,
                         "bytes_per_ant_step": bytes_per_step,
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                            "of one launch, captured separately")
                         if args.workload in CONSTRUCT_DRAM_BYTES_PER_LAUNCH else None},
            "roofline_update": roof_upd,
            "e2e": {"value": e2e, "unit": "ant-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "step": f"one solve through the C ABI on a reused context: upload, "
                            f"candidates, {wl['e2e_epochs']} epochs, download of the best "
                            "routes"},
            "clocks": clk.summary(),
        }
        if roof_upd_hbm is not None:
            line["roofline_update_hbm"] = roof_upd_hbm
        if roof_seq_hbm is not None:
            line["roofline_seq_update_hbm"] = roof_seq_hbm
        if world == 1 and args.workload == "n1000" and not args.no_extras:
            line.update(default_extras(local, torch, _native))
            line["other_configs"] = other_configs(local, torch, _native, args.no_cpu_baseline)
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(inst, m, cand_k=k)
            except Exception as exc:  # reported, not fatal
                line["cpu_baseline"] = {"error": str(exc)[:200]}
        if world == 1 and args.cli and os.path.exists(OUR_CLI):
            # This library's drop-in CLI under the reference's CLI contract,
            # comparable with the reference arm's reference_cuda_same_gpu.
            try:
                line["cli_same_contract"] = cli_epoch_rate(OUR_CLI, inst, m)
                # the reference CUDA kernel's depot-close rule, for a cost
                # comparison with reference_cuda_same_gpu
                line["cli_same_contract_cuda_ref_rule"] = cli_epoch_rate(
                    OUR_CLI, inst, m, extra_env={"ACO_CUDA_DEPOT_RULE": "cuda_ref"})
            except Exception as exc:  # reported, not fatal
                line["cli_same_contract"] = {"error": str(exc)[:200]}
    ctx.close()
    return line


def run_sharded(args, rank, world, local, torch, dist, _native):
    """One colony split over the ranks: m ants per rank, one packet
    all-gather per epoch (NCCL) inside the timed region."""
    from vehicleroutingproblem_b200 import sharding as S
    wl = WORKLOADS[args.workload]
    inst = wl["factory"]()
    n, K, m, k = inst.n, inst.vehicles, wl["ants"], wl["cand_k"]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    col = S.ShardedColony(inst, m, local, stream=stream, cand_k=k, seed=1234)
    col.enqueue_epochs(args.warmup)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    steps0 = col.state().total_steps
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        dev_ms = timed_steps(torch, stream, args.steps, col.enqueue_epoch, flush)
        wall = time.perf_counter() - wall0
    dist.barrier()
    st = col.state()
    assert st.error == 0 and st.epochs == args.warmup + args.steps
    steps_all = float(st.total_steps - steps0)  # every rank's ants (packets carry them)
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_ms_max = float(t[0])
    value = steps_all / (dev_ms_max / 1e3)
    # Per-kernel times of this rank's epoch (plain path, local ants, after
    # the timed region).
    kms = col.ctx.profile_epochs(32) / 32.0
    col.close()

    e2e_vals = []
    h2d = (n + 1) * (8 + 4) + 4095 * 4 + 2 * 256 * 4
    d2h = (n + 2 * K) * 4 + K * 4
    c2 = None
    for i in range(args.e2e_steps):
        dist.barrier()
        t0 = time.perf_counter()
        if c2 is None:
            c2 = S.ShardedColony(inst, m, local, cand_k=k, seed=99 + i,
                                 fixed_epochs=wl["e2e_epochs"])
        else:  # one colony per rank serves every solve (buffers reused)
            c2.setup(inst, cand_k=k, seed=99 + i, fixed_epochs=wl["e2e_epochs"])
        s2 = c2.run(wl["e2e_epochs"])
        c2.best()
        dt = time.perf_counter() - t0
        td = torch.tensor([dt], dtype=torch.float64, device="cuda")
        dist.all_reduce(td, op=dist.ReduceOp.MAX)
        if i > 0:
            e2e_vals.append(s2.total_steps / float(td[0]))
    if c2 is not None:
        c2.close()
    e2e = statistics.median(e2e_vals) if e2e_vals else None

    peak, peak_kind = load_peaks()
    bytes_per_step = k * (4 + 4 + 1)
    local_steps_per_epoch = steps_all / args.steps / world
    achieved = bytes_per_step * local_steps_per_epoch / (float(kms[1]) / 1e3) / 1e9
    if rank != 0:
        return None
    packet_bytes = 4 * S.packet_ints(n, K)
    line = {
        "metric": "ant-steps/s", "value": value, "unit": "ant-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "int32 weights + u8 pheromone (f64 route costs)",
        "data": "synthetic",
        "config": {"workload": wl["name"], "n": n, "K": K, "capacity": inst.capacity,
                   "ants": m * world, "ants_per_gpu": m, "cand_k": k, "step": "one epoch",
                   "l2": "flushed between timed steps (256 MiB write outside the events)",
                   "parallelism": f"one colony split over {world} GPU(s), packet all-gather "
                                  f"({packet_bytes} B per rank) per epoch"},
        "wall_s": wall,
        "gpu_launches": 5 * args.steps,
        "kernels_us": {"weights": float(kms[0]) * 1e3, "construct": float(kms[1]) * 1e3,
                       "evaporate (beside construct in the graph)": float(kms[2]) * 1e3,
                           "best_deposit": float(kms[3]) * 1e3},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": CONSTRUCT_DRAM_BYTES_PER_LAUNCH.get(args.workload),
                     "kernel": "k_construct", "peak_kind": peak_kind,
                     "bytes_per_ant_step": bytes_per_step},
        "e2e": {"value": e2e, "unit": "ant-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "step": f"one split-colony solve on reused colonies: upload, candidates, "
                        f"{wl['e2e_epochs']} epochs with packet exchange, download of the "
                        "best routes"},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(inst, m, cand_k=k)
        except Exception as exc:  # reported, not fatal
            line["cpu_baseline"] = {"error": str(exc)[:200]}
    return line


def batched_measure(torch, local, _native, insts, seed0, steps, warmup, e2e_steps,
                    looped_sample, dist=None, world=1):
    """The batched solver on `insts` (instance i solved with seed seed0 + i):
    autotuned candidate length and shape, `steps` solves timed with CUDA
    events on one stream (L2 flushed between them), the end-to-end rate
    through the C ABI with host buffers on one reused batch object, and the
    single-instance solver looped over a sample of the same instances
    (scaled by n + K)."""
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    b = _native.Batch(local)
    b.set_stream(stream.cuda_stream)
    b.setup(insts, ants=BATCHED["ants"], cand_k=BATCHED["cand_k"], seed=seed0,
            epochs=BATCHED["epochs"])
    # The autotuner picks the candidate-list length (fastest within 0.5 % of
    # the best mean final cost), then the launch shape.
    k, chosen, per_k, trials = b.autotune_k(ks=(16, 20, 32), quality_tol=0.005, trial_epochs=3)
    for _ in range(warmup):
        b.enqueue()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    if dist is not None and world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        dev_ms = timed_steps(torch, stream, steps, b.enqueue, flush)
        wall = time.perf_counter() - wall0
    if dist is not None and world > 1:
        dist.barrier()
    costs, epochs, ant_steps = b.costs()
    assert np.all(epochs == BATCHED["epochs"])
    b.close()
    del flush

    # End to end through the C ABI with host buffers, as a service solving a
    # stream of batches on one batch object: set-up (upload, k-NN; the
    # device buffers of the previous batch are reused), one solve, download
    # of every cost and best route.
    e2e_vals = []
    with _native.Batch(local) as b2:
        for i in range(e2e_steps):
            t0 = time.perf_counter()
            b2.setup(insts, ants=BATCHED["ants"], cand_k=k, seed=seed0,
                     epochs=BATCHED["epochs"])
            b2.set_tuning(*chosen)
            b2.solve()
            res = b2.best_all()
            dt = time.perf_counter() - t0
            assert len(res) == len(insts)
            if i > 0:
                e2e_vals.append(len(insts) / dt)
    # Looping the single-instance solver over a sample, scaled by work.
    looped = None
    if looped_sample > 0:
        sample = list(range(0, len(insts), max(1, len(insts) // looped_sample)))
        t0 = time.perf_counter()
        for i in sample:
            with _native.Context(local) as ctx:
                ctx.setup_instance(insts[i], ants=BATCHED["ants"], cand_k=k,
                                   seed=seed0 + i, fixed_epochs=BATCHED["epochs"])
                ctx.run(BATCHED["epochs"])
                ctx.best()
        ts = time.perf_counter() - t0
        w = np.array([x.n + x.vehicles for x in insts], float)
        t_all = ts * w.sum() / w[sample].sum()
        looped = {"value": len(insts) / t_all, "unit": "instances/s",
                  "sample": f"{len(sample)} instances solved one after another with the "
                            "single-instance C ABI (300 epochs each, set-up and download "
                            "included), scaled by n+K"}
    per_k = {str(kk): {"solve_ms": v[0], "instances_per_s": len(insts) / (v[0] / 1e3),
                       "mean_final_cost": v[1], "solved": v[2]} for kk, v in per_k.items()}
    return {"dev_ms": dev_ms, "wall": wall, "clk": clk.summary(), "chosen": chosen,
            "cand_k": k, "per_k": per_k, "trials": trials, "count": len(insts),
            "ant_steps": float(ant_steps.sum()),
            "mean_cost": float(np.mean(costs[costs < 1e300])) if np.any(costs < 1e300) else None,
            "e2e": statistics.median(e2e_vals) if e2e_vals else None, "looped": looped}


def batched_h2d_d2h(insts):
    """Bytes copied per end-to-end batched step: coordinates (8 B) and
    demands (4 B) per node, an 80-byte descriptor, row offset and size
    (12 B) and two queue orders (8 B) per instance, the level and weight
    tables (256 + 256 ints) and the 4095 eta thresholds up; every best route
    slot (n + 2K ints), the route lengths (K ints) and the costs (8 B) down."""
    nodes = sum(x.n + 1 for x in insts)
    h2d = nodes * 12 + len(insts) * (80 + 12 + 8) + 2048 + 4095 * 4
    d2h = sum((x.n + 2 * x.vehicles) * 4 + x.vehicles * 4 + 8 for x in insts)
    return h2d, d2h


def run_batched(args, rank, world, local, torch, dist, _native):
    insts_all = I.batched_instances(BATCHED["count"], BATCHED["seed0"])
    from vehicleroutingproblem_b200 import sharding as S
    # this rank's share, balanced by the ant-steps per epoch, m (n + K)
    mine = S.split_instances([x.n + x.vehicles for x in insts_all], world)[rank]
    insts = [insts_all[i] for i in mine]
    r = batched_measure(torch, local, _native, insts, BATCHED["seed0"], args.steps, args.warmup,
                        args.e2e_steps, args.looped_sample if rank == 0 else 0, dist, world)
    t = torch.tensor([r["dev_ms"], float(len(insts)), r["ant_steps"]], dtype=torch.float64,
                     device="cuda")
    if world > 1:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:3], op=dist.ReduceOp.SUM)
    dev_ms_max, count_all, steps_all = float(t[0]), float(t[1]), float(t[2])
    value = count_all * args.steps / (dev_ms_max / 1e3)
    ant_steps_s = steps_all * args.steps / (dev_ms_max / 1e3)
    e2e = r["e2e"]
    if world > 1:
        te = torch.tensor([e2e or 0.0], dtype=torch.float64, device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.SUM)
        e2e = float(te[0])
    h2d, d2h = batched_h2d_d2h(insts)
    if rank != 0:
        return None
    chosen = r["chosen"]
    peak, peak_kind = load_peaks()
    bytes_per_step = r["cand_k"] * (4 + 4 + 1)
    achieved = bytes_per_step * ant_steps_s / 1e9
    line = {
        "metric": "instances/s", "value": value, "unit": "instances/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "int32 weights + u8 pheromone (f64 route costs)", "data": "synthetic",
        "config": {"workload": BATCHED["name"], "instances": BATCHED["count"],
                   "step": "one solve of the whole batch (one persistent launch)",
                   "tuning": {"cand_k": r["cand_k"], "lanes_per_ant": chosen[0],
                              "ants_per_block": chosen[1],
                              "order": "largest first" if chosen[2] else "as given"},
                   "autotune_cand_k": r["per_k"],
                   "autotune_trial_ms": [round(float(x), 3) for x in r["trials"]],
                   "l2": "flushed between timed steps (256 MiB write outside the events)",
                   "parallelism": f"instances split over {world} GPUs" if world > 1 else "1 GPU"},
        "ant_steps_per_s": ant_steps_s,
        "wall_s": r["wall"], "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "k_batch_solve",
                     "peak_kind": peak_kind, "bytes_per_ant_step": bytes_per_step},
        "e2e": {"value": e2e, "unit": "instances/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "step": "set-up of the batch through the C ABI, one solve, download of "
                        "every cost and best route"},
        "looped_single_instance": r["looped"],
        "clocks": r["clk"],
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_batched(insts)
        except Exception as exc:
            line["cpu_baseline"] = {"error": str(exc)[:200]}
    return line


LEARNED = dict(train=4096, heldout=256, elite_ants=64, elite_k=16, elite_epochs=120,
               train_epochs=10, batch=4096, lr=2e-3, gammas=(2.0, 4.0, 6.0), validation=8,
               control_betas=(3.0, 5.0, 8.0),
               epochs=300, ants=256, cand_k=32,
               name="learned prior: 4096 training instances n~U[200,1000] (seed 40000), "
                    "256 held-out n=1000 K=8 (seeds 50000-50255), 256 ants 32-NN, "
                    "300 epochs, target = plain final cost +0.5%")
# Useful FLOPs per candidate edge of one training step: forward
# 2 (8*64 + 64*64 + 64), backward 2 (64*64 + 64*64 + 8*64 + 64).
TRAIN_FLOPS_PER_EDGE = 2 * (8 * 64 + 64 * 64 + 64) + 2 * (64 * 64 + 64 * 64 + 8 * 64 + 64)


def learned_measure(local, torch, _native, ntrain, nheld, nval, elite_beta=2.0,
                    residual_beta=None, gammas=None):
    """The learned prior's whole pipeline on one GPU: elite routes of the
    plain batched solver on `ntrain` training instances, the training set,
    tensor-core training, gamma for the learned levels and the beta of a
    control (the plain solver with a sharper hand-set eta^beta) each chosen
    on `nval` validation instances by mean final cost relative to the plain
    solver, then time-to-cost on `nheld` held-out n=1000 instances.
    elite_beta: eta^beta of the plain solver that makes the elite routes;
    residual_beta: the learned levels are added to plain eta^residual_beta
    levels (None: they replace the plain levels)."""
    from vehicleroutingproblem_b200 import prior as PR
    L = LEARNED
    gammas = gammas or L["gammas"]
    tr = I.prior_training_instances(ntrain)
    t0 = time.perf_counter()
    sols = PR.elite_solutions(tr, ants=L["elite_ants"], cand_k=L["elite_k"],
                              epochs=L["elite_epochs"], beta=elite_beta)
    elite_s = time.perf_counter() - t0
    pr = _native.Prior(local, seed=1)
    try:
        t0 = time.perf_counter()
        count = pr.set_dataset(tr, [(x[0], x[1]) for x in sols], cand_k=L["cand_k"])
        dataset_s = time.perf_counter() - t0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        losses = pr.train(L["train_epochs"], batch=L["batch"], lr=L["lr"], seed=11)
        train_s = time.perf_counter() - t0
        val = [I.uniform_instance(1000, 8, 60000 + i) for i in range(nval)]
        base = PR.final_costs(val, L["epochs"], ants=L["ants"], cand_k=L["cand_k"])
        res_kw = ({} if residual_beta is None else
                  {"residual": True, "beta": residual_beta})
        scores = {g: float(np.mean(PR.final_costs(val, L["epochs"], pr, g, ants=L["ants"],
                                                  cand_k=L["cand_k"], **res_kw) / base))
                  for g in gammas}
        gamma = min(scores, key=lambda g: scores[g])
        ctrl = {b: float(np.mean(PR.final_costs(val, L["epochs"], beta=b, ants=L["ants"],
                                                cand_k=L["cand_k"]) / base))
                for b in L["control_betas"]}
        beta_c = min(ctrl, key=lambda b: ctrl[b])
        held = I.prior_heldout_instances(nheld)
        t0 = time.perf_counter()
        res = PR.time_to_cost(held, pr, gamma=gamma, epochs=L["epochs"], ants=L["ants"],
                              cand_k=L["cand_k"], control_beta=beta_c,
                              residual_beta=residual_beta)
        eval_s = time.perf_counter() - t0
    finally:
        pr.close()
    flops = TRAIN_FLOPS_PER_EDGE * 32.0 * count * L["train_epochs"]
    return {"res": res, "gamma": gamma, "scores": scores, "beta_c": beta_c, "ctrl": ctrl,
            "count": count, "losses": losses, "elite_s": elite_s, "dataset_s": dataset_s,
            "train_s": train_s, "eval_s": eval_s, "flops": flops}


def run_learned(args, rank, world, local, torch, dist, _native):
    """Time-to-cost of the learned prior against plain eta on held-out
    instances (one GPU; the whole pipeline runs inside this call)."""
    if rank != 0:
        return None
    L = LEARNED
    ntrain = args.prior_train or L["train"]
    nheld = args.prior_heldout or L["heldout"]
    gammas = tuple(float(x) for x in args.prior_gammas.split(",")) if args.prior_gammas else None
    r = learned_measure(local, torch, _native, ntrain, nheld, L["validation"],
                        elite_beta=args.prior_elite_beta, residual_beta=args.prior_residual_beta,
                        gammas=gammas)
    res = r["res"]
    rows = res.pop("rows")
    peak, peak_kind = None, "fallback"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])  # burst: short launches
        peak_kind = "measured"
    except Exception:
        peak = 1590.0
    achieved = r["flops"] / r["train_s"] / 1e12
    line = {
        "metric": "time-to-cost ratio (learned / plain eta)", "value": res["time_ratio_of_sums"],
        "unit": "ratio", "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 MLP (fp32 accumulate) + int32 weights + u8 pheromone",
        "data": "synthetic",
        "config": {"workload": L["name"], "train_instances": ntrain, "heldout": nheld,
                   "elite_beta": args.prior_elite_beta,
                   "levels": ("learned, replacing plain eta" if args.prior_residual_beta is None
                              else f"learned, added to plain eta^{args.prior_residual_beta:g}"),
                   "gamma": r["gamma"], "gamma_validation_final_cost": r["scores"],
                   "control_beta": r["beta_c"], "control_validation_final_cost": r["ctrl"]},
        "time_to_cost": res,
        "training": {"examples": r["count"], "epochs": L["train_epochs"], "batch": L["batch"],
                     "lr": L["lr"],
                     "loss_first_last": [float(r["losses"][0]), float(r["losses"][-1])],
                     "elite_s": r["elite_s"], "dataset_s": r["dataset_s"], "train_s": r["train_s"],
                     "examples_per_s": r["count"] * L["train_epochs"] / r["train_s"]},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "k_prior_mlp<train> with reduce, Adam and the per-epoch "
                               "shuffle upload (host-timed)",
                     "flops_per_edge": TRAIN_FLOPS_PER_EDGE},
        "eval_s": r["eval_s"],
        "per_instance_sample": rows[:4],
    }
    return line


def other_configs(local, torch, _native, no_cpu):
    """The two other single-instance configurations the CPU comparison is
    quoted on, on bounded samples: the small n=100 and the clustered n=2000
    workloads, device ant-steps/s over 50 epochs (CUDA events, L2 flushed
    between epochs) beside the reference's OpenMP solver on the host cores."""
    out = {}
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    for name in ("small", "clustered2000"):
        wl = WORKLOADS[name]
        inst = wl["factory"]()
        try:
            with _native.Context(local) as ctx:
                ctx.set_stream(stream.cuda_stream)
                ctx.setup_instance(inst, ants=wl["ants"], cand_k=wl["cand_k"], seed=1234)
                ctx.enqueue_epochs(5)
                torch.cuda.synchronize()
                s0 = ctx.state().total_steps
                steps = 50
                ms = timed_steps(torch, stream, steps, lambda: ctx.enqueue_epochs(1), flush)
                done = ctx.state().total_steps - s0
            r = {"workload": wl["name"], "value": done / (ms / 1e3), "unit": "ant-steps/s",
                 "ms_per_step": ms / steps, "steps": steps, "warmup": 5}
            if not no_cpu:
                r["cpu_baseline"] = cpu_baseline(inst, wl["ants"], target_s=6.0,
                                                 cand_k=wl["cand_k"])
                r["vs_cpu_baseline"] = r["value"] / r["cpu_baseline"]["value"]
            out[name] = r
        except Exception as exc:  # reported, not fatal
            out[name] = {"error": str(exc)[:300]}
    return out


def default_extras(local, torch, _native):
    """The other two figures of the headline metric, on bounded samples so
    that the default run stays within a few minutes: instances/s of the
    batched form (the full 512-instance batch) against looping the plain
    single-instance solver, and the learned prior's time-to-cost against
    plain eta on a small held-out set, with the tuned-beta control."""
    out = {}
    insts = I.batched_instances(BATCHED["count"], BATCHED["seed0"])
    try:
        r = batched_measure(torch, local, _native, insts, BATCHED["seed0"], steps=3, warmup=1,
                            e2e_steps=2, looped_sample=8)
        value = r["count"] * 3 / (r["dev_ms"] / 1e3)
        looped = r["looped"]
        out["batched"] = {
            "metric": "instances/s", "value": value, "unit": "instances/s",
            "workload": BATCHED["name"], "steps": 3, "warmup": 1,
            "ms_per_step": r["dev_ms"] / 3, "e2e": r["e2e"],
            "tuning": {"cand_k": r["cand_k"], "lanes_per_ant": r["chosen"][0],
                       "ants_per_block": r["chosen"][1],
                       "order": "largest first" if r["chosen"][2] else "as given"},
            "autotune_cand_k": r["per_k"],
            "looped_single_instance": looped,
            "vs_looped": value / looped["value"] if looped else None,
            "mean_final_cost": r["mean_cost"], "clocks": r["clk"]}
    except Exception as exc:  # reported, not fatal
        out["batched"] = {"error": str(exc)[:300]}
    try:
        L = LEARNED
        ntrain, nheld, nval = 512, 8, 4
        r = learned_measure(local, torch, _native, ntrain, nheld, nval)
        res = r["res"]
        res.pop("rows")
        out["learned_time_to_cost"] = {
            "metric": "time-to-cost ratio (learned / plain eta)",
            "value": res["time_ratio_of_sums"], "unit": "ratio", "higher_is_better": False,
            "workload": (f"learned prior: {ntrain} training instances n~U[200,1000], {nheld} "
                         f"held-out n=1000 K=8 (seeds 50000-{50000 + nheld - 1}), {nval} "
                         f"validation, 256 ants 32-NN, {L['epochs']} epochs, target = plain "
                         "final cost +0.5%"),
            "gamma": r["gamma"], "control_beta": r["beta_c"], "time_to_cost": res,
            "train_s": r["train_s"], "pipeline_s": r["elite_s"] + r["dataset_s"] +
            r["train_s"] + r["eval_s"]}
    except Exception as exc:  # reported, not fatal
        out["learned_time_to_cost"] = {"error": str(exc)[:300]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="n1000",
                    choices=sorted(WORKLOADS) + ["batched", "learned", "costdist"])
    ap.add_argument("--costdist-seeds", type=int, default=12,
                    help="costdist: seeds per solver")
    ap.add_argument("--costdist-seconds", type=float, default=2.0,
                    help="costdist: wall-time limit of each run")
    ap.add_argument("--prior-train", type=int, default=None,
                    help="learned: training instances (default 4096)")
    ap.add_argument("--prior-heldout", type=int, default=None,
                    help="learned: held-out instances (default 256)")
    ap.add_argument("--prior-elite-beta", type=float, default=2.0,
                    help="learned: eta^beta of the plain solver making the elite routes")
    ap.add_argument("--prior-residual-beta", type=float, default=None,
                    help="learned: add the learned levels to plain eta^beta levels")
    ap.add_argument("--prior-gammas", default=None,
                    help="learned: comma-separated gammas to choose from on validation")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--looped-sample", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="n1000: skip the batched and learned-prior figures added to the line")
    ap.add_argument("--no-large-update", action="store_true",
                    help="skip the n=16000 pheromone-sweep roofline of small workloads")
    ap.add_argument("--no-cli", dest="cli", action="store_false",
                    help="skip the drop-in CLI timing on the unit-demand twin")
    ap.add_argument("--colony", default="auto", choices=["auto", "sharded"],
                    help="single-instance workloads: auto = one GPU runs the plain "
                         "graph-launched epochs, several GPUs split the colony")
    args = ap.parse_args()
    batched = args.workload == "batched"
    if args.steps is None:
        args.steps = 3 if batched else 2000
    if args.warmup is None:
        args.warmup = 3 if batched else 20
    if args.e2e_steps is None:
        args.e2e_steps = 3 if batched else 8
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()
    if args.workload == "costdist":
        return run_costdist(args) if rank == 0 else 0

    if args.impl == "reference":
        if args.workload == "learned":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no learned prior; its plain eta solver is "
                                  "the denominator of this workload's ratio"}), flush=True)
            return 0
        return run_reference_arm(args, rank, world)

    import datetime

    import torch
    import torch.distributed as dist
    from vehicleroutingproblem_b200 import _native

    torch.cuda.set_device(local)
    learned = args.workload == "learned"
    sharded = not batched and not learned and (world > 1 or args.colony == "sharded")
    pg = world > 1 or sharded
    if world > 1 or (pg and "MASTER_ADDR" in os.environ and "WORLD_SIZE" in os.environ):
        # launched by torchrun (its rendezvous variables are set)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif pg:
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                                world_size=1, timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    try:
        fn = (run_batched if batched else run_learned if learned else
              run_sharded if sharded else run_single)
        line = fn(args, rank, world, local, torch, dist, _native)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
