"""Reference-CUDA depot rule (ACO_CUDA_DEPOT_RULE=cuda_ref, depot_rule=1):
the device tables and routes against the oracle's restatement of the rule,
and the CLI switch."""
import os
import subprocess

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _roomy(n, K, seed, cap_frac, unit=True):
    """Capacity well above need, so routes may close early."""
    base = I.uniform_instance(n, K, seed)
    if unit:
        base = base.unit_twin()
    cap = int(np.ceil(base.demand.sum() / (cap_frac * K)))
    return I.Instance(base.name + "_roomy", base.x, base.y, base.demand, K, cap)


CASES = {
    "unit_roomy": (lambda: _roomy(200, 4, 701, 0.75), 32, 64),
    "unit_twin": (lambda: I.uniform_instance(300, 5, 702).unit_twin(), 32, 48),
    "demand_roomy": (lambda: _roomy(250, 5, 703, 0.6, unit=False), 20, 48),
    "n1000_unit": (lambda: I.workload_n1000().unit_twin(), 32, 32),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_ref_rule_matches_oracle(native, oracle_mod, name):
    O = oracle_mod
    make, k, m = CASES[name]
    inst = make()
    n, K = inst.n, inst.vehicles
    demand = None if inst.is_unit_demand() else inst.demand
    rs = np.random.RandomState(7)
    tau = rs.randint(60, 256, size=(n + 1) ** 2).astype(np.uint8)
    with native.Context(0) as c:
        c.setup_instance(inst, ants=m, cand_k=k, seed=31, depot_rule=1)
        c.set_tau(tau)
        c.construct(5)
        cand, lvl = c.candidates()
        A, lut, thr = O.tables()
        lvl0, rdep, e_dep = c.depot_tables()
        d2 = ((inst.x - inst.x[0]) ** 2 + (inst.y - inst.y[0]) ** 2).astype(np.float32)
        exp_lvl0 = np.array([O.lib().orc_level(float(v), thr.ctypes.data_as(
            __import__("ctypes").c_void_p), len(thr)) for v in d2], np.uint16)
        assert np.array_equal(lvl0, exp_lvl0)
        assert np.array_equal(rdep, O.depot_rel(n, c.k, cand, lvl, tau, A, lvl0, e_dep))
        w = O.weights(n, c.k, cand, lvl, tau, A, lut)
        nodes, lens, cost, feas, steps, draws = c.ants()
        differs = 0
        for a in range(m):
            of, on, ol, oc, os_, od = O.construct_ant(
                inst.x, inst.y, demand, K, inst.capacity, c.k, cand, w, 31, 5, a,
                rule=1, rdep=rdep, lut=lut)
            assert np.array_equal(lens[a], ol), (a, lens[a], ol)
            assert np.array_equal(nodes[a][: ol.sum()], on)
            assert cost[a] == oc and bool(feas[a]) == of and steps[a] == os_ and draws[a] == od
            sf, sn, sl, *_ = O.construct_ant(inst.x, inst.y, demand, K, inst.capacity, c.k,
                                             cand, w, 31, 5, a)
            differs += int(not np.array_equal(sl, ol) or not np.array_equal(sn, on))
        assert differs > 0  # the rule changes routes
        st = c.run(12)
        assert st.error == 0 and st.epochs == 12 and np.isfinite(st.global_best)


def test_cli_depot_rule_switch(tmp_path):
    inst = _roomy(120, 5, 704, 0.75)
    vrp = tmp_path / "r.vrp"
    I.write_vrp(inst, str(vrp))
    cli = os.path.join(ROOT, "aco_vrp_cuda.out")
    out = {}
    for rule in ("seq", "cuda_ref"):
        env = dict(os.environ, ACO_SOLVER_FIXED_EPOCHS="30", ACO_SOLVER_STAGNATION_EPOCHS="0",
                   ACO_SOLVER_PROGRESS_INTERVAL_SECONDS="0", ACO_CUDA_DEPOT_RULE=rule)
        r = subprocess.run([cli, str(vrp), "5", "32", "3"], env=env, capture_output=True,
                           text=True, timeout=120)
        assert r.returncode == 0 and "best cost:" in r.stdout, r.stderr
        assert "not recognised" not in r.stderr
        out[rule] = r.stdout.split("best cost:")[1].strip()
        routes = [ln for ln in r.stdout.splitlines() if ln.startswith("Route")]
        served = sorted(int(t) for ln in routes for t in ln.split(":")[1].split())
        assert served == list(range(1, inst.n + 1))
    assert out["seq"] != out["cuda_ref"]
