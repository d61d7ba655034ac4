"""Generates the golden construct fixtures from the reference's own code.

Run from the repository root after ``make -C oracle all ref`` (needs the
reference sources to build ``oracle/_ref/libseqref.so``):

    python tests/golden/make_golden.py

For each case the candidate lists come from the oracle's k-NN, the integer
weights from the oracle's weight rule over a seeded pheromone matrix, and the
draws from the counter-based stream; the routes, lengths, costs and draw
counts are what the reference's build_ant_solution
(src/seq/aco_sequential.c:616-681) produces from them.  The reference only
accepts unit demand, so all cases are unit-demand.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from vehicleroutingproblem_b200 import instances as I  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def smoke_instance() -> I.Instance:
    # The reference smoke test's 8-customer instance (tools/bash/smoke_test.sh:17-48).
    xs = np.array([50, 10, 20, 10, 20, 80, 90, 80, 90], np.float32)
    ys = np.array([50, 10, 10, 20, 20, 80, 80, 90, 90], np.float32)
    d = np.ones(9, np.int32)
    d[0] = 0
    return I.Instance("smoke", xs, ys, d, 2, 5)


CASES = [
    # name, instance factory, k, ants, tau mode, seed, epoch
    ("smoke_k8", smoke_instance, 8, 16, "init", 1234, 0),
    ("u60_k3", lambda: I.uniform_instance(60, 3, 501).unit_twin(), 20, 24, "random", 77, 3),
    ("u200_k4", lambda: I.uniform_instance(200, 4, 502).unit_twin(), 32, 24, "random", 1234, 11),
    ("c300_k5", lambda: I.clustered_instance(300, 5, 503).unit_twin(), 32, 16, "random", 9, 0),
    ("u120_k6_tight", lambda: I.uniform_instance(120, 6, 504).unit_twin(), 16, 16, "sparse", 5, 2),
]


def make_tau(n: int, mode: str, seed: int, q0: int) -> np.ndarray:
    rs = np.random.RandomState(seed + 17)
    if mode == "init":
        return np.full((n + 1) * (n + 1), q0, np.uint8)
    if mode == "random":
        return rs.randint(0, 256, size=(n + 1) * (n + 1)).astype(np.uint8)
    t = np.zeros((n + 1) * (n + 1), np.uint8)  # mostly q_min with a few strong arcs
    idx = rs.randint(0, t.size, size=t.size // 20)
    t[idx] = rs.randint(150, 256, size=idx.size).astype(np.uint8)
    return t


def main() -> None:
    O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libseqref.so missing: run `make -C oracle ref`")
    P = O.params()
    A, lut, thr = O.tables(1.0, 2.0, P["log_tau_step"])
    for name, factory, k, ants, mode, seed, epoch in CASES:
        inst = factory()
        n, K, cap = inst.n, inst.vehicles, inst.capacity
        k = min(k, n)
        cand = O.knn(inst.x, inst.y, k)
        lvl = O.levels(inst.x, inst.y, cand, k, thr)
        tau = make_tau(n, mode, seed, P["q_tau0"])
        w = O.weights(n, k, cand, lvl, tau, A, lut)
        R = n + 2 * K
        nodes = np.zeros((ants, R), np.int32)
        lens = np.zeros((ants, K), np.int32)
        costs = np.zeros(ants, np.float64)
        used = np.zeros(ants, np.int32)
        for ant in range(ants):
            ds = O.draws(seed, epoch, ant, 0, n + K + 1)
            rn, rl, rc, ru = O.ref_construct_ant(inst.x, inst.y, K, cap, k, cand, w, ds)
            nodes[ant, : rn.size] = rn
            lens[ant] = rl
            costs[ant] = rc
            used[ant] = ru
        path = os.path.join(OUT, f"construct_{name}.npz")
        np.savez_compressed(path, x=inst.x, y=inst.y, K=K, cap=cap, k=k, seed=seed,
                            epoch=epoch, cand=cand, lvl=lvl, tau=tau, w=w, nodes=nodes,
                            lens=lens, costs=costs, draws_used=used)
        print(f"{path}: n={n} K={K} cap={cap} k={k} ants={ants} "
              f"mean cost {costs.mean():.3f}")


if __name__ == "__main__":
    main()
