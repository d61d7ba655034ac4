"""Edge cases of the construction and the epoch loop on the GPU against the
oracle: one customer, one vehicle, customers that cannot be served (no
feasible ant: the epoch changes no pheromone), duplicate points, more
vehicles than customers."""
import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu


def _inst(name, xy, dem, K, cap):
    x = np.array([p[0] for p in xy], np.float32)
    y = np.array([p[1] for p in xy], np.float32)
    d = np.array(dem, np.int32)
    return I.Instance(name, x, y, d, K, cap)


def _edges():
    rs = np.random.RandomState(5)
    pts = [(500, 500)] + [tuple(rs.randint(0, 1001, 2)) for _ in range(60)]
    dup = [(500, 500)] + [(100, 100)] * 10 + [(900, 900)] * 10 + [tuple(rs.randint(0, 1001, 2))
                                                              for _ in range(20)]
    return {
        "one_customer": _inst("one", [(500, 500), (10, 20)], [0, 3], 1, 5),
        "one_vehicle": _inst("onev", pts, [0] + [1] * 60, 1, 60),
        "more_vehicles_than_customers": _inst("mv", pts[:6], [0, 2, 2, 2, 2, 2], 9, 2),
        "duplicates": _inst("dup", dup, [0] + [1] * 40, 4, 12),
        # customer 60 needs 61 of a capacity of 60: no ant can serve it
        "unservable": _inst("big", pts, [0] + [5] * 59 + [61], 6, 60),
    }


@pytest.mark.parametrize("name", sorted(_edges()))
def test_edge_construct_matches_oracle(native, oracle_mod, name):
    O = oracle_mod
    inst = _edges()[name]
    n, K = inst.n, inst.vehicles
    k = min(8, n)
    demand = None if inst.is_unit_demand() else inst.demand
    with native.Context(0) as c:
        c.setup_instance(inst, ants=12, cand_k=k, seed=17)
        cand, lvl = c.candidates()
        A, lut, _ = O.tables()
        tau = c.tau()
        w = O.weights(n, c.k, cand, lvl, tau, A, lut)
        c.construct(0)
        nodes, lens, cost, feas, steps, draws = c.ants()
        for a in range(12):
            f, on, ol, oc, os_, od = O.construct_ant(inst.x, inst.y, demand, K, inst.capacity,
                                                     c.k, cand, w, 17, 0, a)
            assert np.array_equal(lens[a], ol) and np.array_equal(nodes[a][: ol.sum()], on)
            assert bool(feas[a]) == f and cost[a] == oc and steps[a] == os_ and draws[a] == od
        if name == "unservable":
            assert not feas.any()
        else:
            assert feas.all()


def test_no_feasible_ant_leaves_pheromone_unchanged(native):
    """With no feasible ant the reference neither evaporates nor deposits
    (src/cuda/aco_cuda.cu:354-399): the pipelined epochs must keep the
    current pheromone buffer."""
    inst = _edges()["unservable"]
    with native.Context(0) as c:
        c.setup_instance(inst, ants=16, cand_k=8, seed=3)
        t0 = c.tau()
        st, recs = c.run(20, want_records=True)
        assert st.epochs == 20 and not st.found and st.iter_since_best == 20
        assert all(not r.found for r in recs)
        assert np.array_equal(c.tau(), t0)
        nodes, lens, cost = c.best()
        assert cost == float("inf") and nodes.size == 0
