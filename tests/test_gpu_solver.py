"""GPU end-to-end tests of the reference-facing entry points: the C solver
aco_vrp_cuda_with_capacity / _with_demands and the drop-in CLI, on the
reference's smoke instance (tools/bash/smoke_test.sh) and on generated
instances.  Validity is checked the way the reference checks its runs:
structure (solution_validate), FP64 cost recomputed from the routes, and
capacity."""
import os
import re
import subprocess

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I
from vehicleroutingproblem_b200 import solver

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "aco_vrp_cuda.out")

SMOKE_X = np.array([50, 10, 20, 10, 20, 80, 90, 80, 90], np.float32)
SMOKE_Y = np.array([50, 10, 10, 20, 20, 80, 80, 90, 90], np.float32)


def check_routes(routes, n, K, x, y, demand=None, cap=None):
    assert len(routes) == K
    seen = []
    for r in routes:
        assert len(r) >= 2 and r[0] == 0 and r[-1] == 0 and 0 not in r[1:-1]
        seen += r[1:-1]
        if demand is not None:
            assert sum(demand[v] for v in r) <= cap
    assert sorted(seen) == list(range(1, n + 1))
    xd, yd = x.astype(np.float64), y.astype(np.float64)
    return sum(float(np.sum(np.hypot(np.diff(xd[r]), np.diff(yd[r])))) for r in routes)


@pytest.fixture
def stag_env(monkeypatch):
    monkeypatch.setenv("ACO_SOLVER_STAGNATION_EPOCHS", "10")
    monkeypatch.setenv("ACO_SOLVER_TIMEOUT_SECONDS", "10")


def test_c_entry_smoke_instance(stag_env, capfd):
    rc, routes, cost = solver.aco_vrp_cuda_with_capacity(8, 2, 5, 16, SMOKE_X, SMOKE_Y, seed=1234)
    assert rc == 0
    ref = check_routes(routes, 8, 2, SMOKE_X, SMOKE_Y)
    assert abs(ref - cost) <= 1e-9 * ref
    out = capfd.readouterr().out
    assert "CUDA Solver starting... (N=8, K=2, M=16)" in out
    assert re.search(r"\[progress\]\[cuda\] epoca=1 \| epoche_rimanenti_prima_stop=\d+ \| "
                     r"tempo_trascorso=\d+\.\ds \| tempo_rimanente=[\d.]+s \| best_cost=[\d.]+", out)


def test_c_entry_demands(stag_env):
    inst = I.uniform_instance(300, 6, 77, demand_max=100)
    rc, routes, cost = solver.aco_vrp_cuda_with_demands(
        inst.n, inst.vehicles, inst.capacity, 64, inst.x, inst.y, inst.demand, seed=5)
    assert rc == 0
    ref = check_routes(routes, inst.n, inst.vehicles, inst.x, inst.y, inst.demand, inst.capacity)
    assert abs(ref - cost) <= 1e-9 * ref


def test_cli_smoke_contract(tmp_path):
    """The reference smoke test's checks (tools/bash/smoke_test.sh:50-72)."""
    from tests.test_boundary import SMOKE
    p = tmp_path / "smoke.vrp"
    p.write_text(SMOKE)
    env = dict(os.environ, ACO_SOLVER_TIMEOUT_SECONDS="10", ACO_SOLVER_STAGNATION_EPOCHS="10")
    r = subprocess.run(["timeout", "60", CLI, str(p), "2", "0", "1234"], capture_output=True,
                       text=True, env=env)
    assert r.returncode == 0, r.stderr
    assert re.search(r"^Cost: [0-9]+([.][0-9]+)?$", r.stdout, re.M)
    assert re.search(r"^best cost: [0-9]+([.][0-9]+)?$", r.stdout, re.M)
    route_lines = [l for l in r.stdout.splitlines() if l.startswith("Route ")]
    assert len(route_lines) == 2
    served = sorted(int(v) for l in route_lines for v in l.split(":")[1].split())
    assert served == list(range(1, 9))


def test_cli_demand_instance(tmp_path):
    inst = I.uniform_instance(200, 5, 31, demand_max=50)
    p = str(tmp_path / "d.vrp")
    I.write_vrp(inst, p)
    env = dict(os.environ, ACO_SOLVER_FIXED_EPOCHS="30")
    r = subprocess.run(["timeout", "120", CLI, p, "5", "64", "9"], capture_output=True,
                       text=True, env=env)
    assert r.returncode == 0, r.stderr
    routes = [[0] + [int(v) for v in l.split(":")[1].split()] + [0]
              for l in r.stdout.splitlines() if l.startswith("Route ")]
    cost = check_routes(routes, inst.n, 5, inst.x, inst.y, inst.demand, inst.capacity)
    printed = float(re.search(r"^best cost: ([0-9.]+)$", r.stdout, re.M).group(1))
    assert abs(printed - cost) <= max(0.1, 1e-4 * cost)  # analyze_results.py:295-297


def test_solve_improves_over_epochs():
    inst = I.workload_small()
    routes, cost, st = solver.solve(inst, ants=128, epochs=60, seed=3, cand_k=20)
    ref = check_routes(routes, inst.n, inst.vehicles, inst.x, inst.y, inst.demand,
                       inst.capacity)
    assert abs(ref - cost) <= 1e-9 * ref and st.epochs == 60
    _, cost1, _ = solver.solve(inst, ants=128, epochs=1, seed=3, cand_k=20)
    assert cost <= cost1
