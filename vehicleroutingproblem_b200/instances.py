"""Seeded CVRP instance generation and TSPLIB ``.vrp`` reading/writing.

The reference ships a generator (``tools/python/generate_vrp_problem.py:7-41``)
that needs the absent ``vrplib`` package and only makes unit-demand instances
on a 100x100 grid.  This module replaces it for the benchmark workloads:

* uniform instances: depot fixed at (500, 500), customers with integer
  coordinates uniform in [0, 1000]^2, integer demands uniform in
  [1, ``demand_max``], and ``Q = ceil(sum(d) / (0.9 K))``;
* clustered instances: depot at the centre, 70% of customers drawn from 8
  isotropic Gaussian clusters (sigma 50, centres uniform in [100, 900]^2), 30%
  uniform; coordinates rounded and clipped to [0, 1000];
* unit-demand twins: same coordinates, demand 1 and
  ``CAPACITY = ceil(n / (0.9 K))`` customers, which the reference binaries can
  load (its parser rejects any demand other than 1,
  ``src/common/instance_parser.c:157-166``).

Draw order (numpy ``RandomState(seed)``; the order is part of the format):

uniform:   ``xy = randint(0, 1001, size=(n, 2))`` then
           ``demand = randint(1, demand_max + 1, size=n)``.
clustered: ``centres = uniform(100, 900, size=(8, 2))``,
           ``nc = int(round(0.7 n))``, ``lab = randint(0, 8, size=nc)``,
           ``noise = normal(0, 50, size=(nc, 2))``,
           ``uni = randint(0, 1001, size=(n - nc, 2))``, ``perm = permutation(n)``
           (applied to the stacked clustered+uniform points), then demands.
batched:   ``n = randint(n_lo, n_hi + 1)`` first, then the uniform draws.

The TSPLIB text follows the layout of the reference's instances
(``instances/generated_benchmark/*.vrp``): NAME, TYPE, DIMENSION (n+1),
VEHICLES, EDGE_WEIGHT_TYPE, CAPACITY, NODE_COORD_SECTION (1-based ids, depot
first), DEMAND_SECTION, DEPOT_SECTION, EOF.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class Instance:
    """A CVRP instance: node 0 is the depot, nodes 1..n are customers."""

    name: str
    x: np.ndarray          # float32 [n+1]
    y: np.ndarray          # float32 [n+1]
    demand: np.ndarray     # int32 [n+1], demand[0] == 0
    vehicles: int
    capacity: int

    @property
    def n(self) -> int:
        return int(self.x.shape[0] - 1)

    def unit_twin(self) -> "Instance":
        """Same coordinates, unit demand, capacity ceil(n / (0.9 K)) customers."""
        n = self.n
        d = np.ones(n + 1, dtype=np.int32)
        d[0] = 0
        cap = int(math.ceil(n / (0.9 * self.vehicles)))
        return Instance(self.name + "_unit", self.x.copy(), self.y.copy(), d,
                        self.vehicles, cap)

    def is_unit_demand(self) -> bool:
        return bool(np.all(self.demand[1:] == 1))


def _capacity(demand: np.ndarray, K: int) -> int:
    return int(math.ceil(float(demand.sum()) / (0.9 * K)))


def _assemble(name: str, xy: np.ndarray, demand: np.ndarray, K: int,
              depot=(500, 500)) -> Instance:
    n = xy.shape[0]
    x = np.empty(n + 1, dtype=np.float32)
    y = np.empty(n + 1, dtype=np.float32)
    x[0], y[0] = depot
    x[1:] = xy[:, 0]
    y[1:] = xy[:, 1]
    d = np.zeros(n + 1, dtype=np.int32)
    d[1:] = demand
    return Instance(name, x, y, d, K, _capacity(d, K))


def uniform_instance(n: int, K: int, seed: int, demand_max: int = 100,
                     name: Optional[str] = None) -> Instance:
    rs = np.random.RandomState(seed)
    xy = rs.randint(0, 1001, size=(n, 2))
    dem = rs.randint(1, demand_max + 1, size=n)
    return _assemble(name or f"u{n}_k{K}_s{seed}", xy, dem, K)


def clustered_instance(n: int, K: int, seed: int, demand_max: int = 100,
                       n_clusters: int = 8, sigma: float = 50.0,
                       frac_clustered: float = 0.7,
                       name: Optional[str] = None) -> Instance:
    rs = np.random.RandomState(seed)
    centres = rs.uniform(100, 900, size=(n_clusters, 2))
    nc = int(round(frac_clustered * n))
    lab = rs.randint(0, n_clusters, size=nc)
    noise = rs.normal(0.0, sigma, size=(nc, 2))
    clus = np.clip(np.rint(centres[lab] + noise), 0, 1000)
    uni = rs.randint(0, 1001, size=(n - nc, 2))
    pts = np.vstack([clus, uni]).astype(np.int64)
    perm = rs.permutation(n)
    pts = pts[perm]
    dem = rs.randint(1, demand_max + 1, size=n)
    return _assemble(name or f"c{n}_k{K}_s{seed}", pts, dem, K)


def batched_instances(count: int = 512, seed0: int = 30000, n_lo: int = 50,
                      n_hi: int = 500, demand_max: int = 100,
                      customers_per_vehicle: int = 60) -> List[Instance]:
    out = []
    for i in range(count):
        seed = seed0 + i
        rs = np.random.RandomState(seed)
        n = int(rs.randint(n_lo, n_hi + 1))
        K = int(math.ceil(n / customers_per_vehicle))
        xy = rs.randint(0, 1001, size=(n, 2))
        dem = rs.randint(1, demand_max + 1, size=n)
        out.append(_assemble(f"b{n}_k{K}_s{seed}", xy, dem, K))
    return out


# --------------------------------------------------------------------------
# The benchmark workloads (sizes and seeds of the five configurations).
# --------------------------------------------------------------------------

def workload_small() -> Instance:
    """n=100, K=4, demands [1,30], seed 1001 (k=20, 128 ants, 200 epochs)."""
    return uniform_instance(100, 4, 1001, demand_max=30, name="c1_n100_k4_s1001")


def workload_n1000() -> Instance:
    """n=1000, K=8, demands [1,100], seed 19001 (k=32, 256 ants)."""
    return uniform_instance(1000, 8, 19001, demand_max=100,
                            name="c2_n1000_k8_s19001")


def workload_clustered2000(seed: int = 29001) -> Instance:
    """n=2000, K=16 clustered, demands [1,100] (k=32, 1024 ants, 500 epochs)."""
    return clustered_instance(2000, 16, seed, demand_max=100,
                              name=f"c3_n2000_k16_s{seed}")


def workload_large(n: int = 16000) -> Instance:
    """Large uniform instance in the reference's published CUDA size range
    (n = 4000-64000): K = n / 1000 vehicles, demands [1,100], seed 10 n + 1
    (n=16000: tau is 256 MB; n=32000: 1 GB; 256 ants, 32-NN)."""
    K = max(1, n // 1000)
    return uniform_instance(n, K, 10 * n + 1, demand_max=100, name=f"large_n{n}_k{K}")


def prior_training_instances(count: int = 4096, seed0: int = 40000) -> List[Instance]:
    """Training set of the learned prior: n ~ U[200,1000] (drawn from seed0),
    K = ceil(n/125), demands [1,100]; even indices uniform, odd clustered;
    instance i uses seed seed0 + 1 + i."""
    rs = np.random.RandomState(seed0)
    ns = rs.randint(200, 1001, size=count)
    out = []
    for i, n in enumerate(ns):
        n = int(n)
        K = int(math.ceil(n / 125))
        make = uniform_instance if i % 2 == 0 else clustered_instance
        out.append(make(n, K, seed0 + 1 + i))
    return out


def prior_heldout_instances(count: int = 256, seed0: int = 50000) -> List[Instance]:
    """Held-out evaluation set of the learned prior: n=1000, K=8, uniform,
    demands [1,100] (the n1000 workload's shape), seeds seed0 .. seed0+count-1."""
    return [uniform_instance(1000, 8, seed0 + i) for i in range(count)]


# --------------------------------------------------------------------------
# TSPLIB text
# --------------------------------------------------------------------------

def _fmt_coord(v: float) -> str:
    f = float(v)
    return str(int(f)) if f.is_integer() else repr(f)


def write_vrp(inst: Instance, path: str) -> None:
    n = inst.n
    lines = [f"NAME: {inst.name}", "TYPE: CVRP", f"DIMENSION: {n + 1}",
             f"VEHICLES: {inst.vehicles}", "EDGE_WEIGHT_TYPE: EUC_2D",
             f"CAPACITY: {inst.capacity}", "NODE_COORD_SECTION"]
    for i in range(n + 1):
        lines.append(f"{i + 1}\t{_fmt_coord(inst.x[i])}\t{_fmt_coord(inst.y[i])}")
    lines.append("DEMAND_SECTION")
    for i in range(n + 1):
        lines.append(f"{i + 1}\t{int(inst.demand[i])}")
    lines += ["DEPOT_SECTION", "1", "-1", "EOF"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_vrp(path: str) -> Instance:
    """Reads the TSPLIB subset the reference parser reads
    (``src/common/instance_parser.c:226-388``), with demands of any value."""
    name = path
    n = K = cap = 0
    xs = ys = dem = None
    with open(path) as f:
        toks = f.read().splitlines()
    i = 0
    while i < len(toks):
        line = toks[i]
        key = line.split(":")[0].strip()
        if line.startswith("NAME"):
            name = line.split(":", 1)[1].strip() if ":" in line else line[4:].strip()
        elif line.startswith("DIMENSION"):
            n = int(line.split(":", 1)[1]) - 1 if ":" in line else int(line.split()[1]) - 1
        elif line.startswith("VEHICLES"):
            K = int(line.split(":", 1)[1]) if ":" in line else int(line.split()[1])
        elif line.startswith("CAPACITY"):
            cap = int(line.split(":", 1)[1]) if ":" in line else int(line.split()[1])
        elif key == "NODE_COORD_SECTION":
            xs = np.empty(n + 1, dtype=np.float32)
            ys = np.empty(n + 1, dtype=np.float32)
            for j in range(n + 1):
                i += 1
                parts = toks[i].split()
                xs[j] = float(parts[1])
                ys[j] = float(parts[2])
        elif key == "DEMAND_SECTION":
            dem = np.empty(n + 1, dtype=np.int32)
            for j in range(n + 1):
                i += 1
                parts = toks[i].split()
                dem[j] = int(parts[1])
        elif key == "DEPOT_SECTION":
            depots = []
            while i + 1 < len(toks) and toks[i + 1].strip() not in ("-1", "EOF"):
                i += 1
                depots.append(int(toks[i].split()[0]))
            if depots and depots != [1]:
                raise ValueError(f"{path}: only node 1 may be the depot (DEPOT_SECTION)")
        i += 1
    if xs is None or dem is None or n <= 0:
        raise ValueError(f"{path}: missing DIMENSION/NODE_COORD_SECTION/DEMAND_SECTION")
    return Instance(name, xs, ys, dem, K, cap)
