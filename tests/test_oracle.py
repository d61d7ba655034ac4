"""CPU tests of the oracle: pinned to the reference's own sequential construct
code (golden fixtures made by tests/golden/make_golden.py, and the live
oracle/_ref harness when it is built) and to published Philox vectors."""
import glob
import os

import numpy as np
import pytest

from vehicleroutingproblem_b200 import instances as I

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "construct_*.npz")))


def test_philox_known_answers(oracle_mod):
    O = oracle_mod
    # Random123 known-answer vectors for Philox4x32-10.
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox([0xffffffff] * 4, [0xffffffff] * 2)) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                         [0xa4093822, 0x299f31d0])) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_draws_are_24_bit_and_addressable(oracle_mod):
    O = oracle_mod
    d = O.draws(1234, 7, 3, 0, 512)
    assert d.max() < (1 << 24)
    assert len(np.unique(d)) > 500
    # draw index d -> word d%4 of block d/4
    blk = O.philox([5, 3, 7, 0], [1234, 0x5EEDC0DE])
    assert [O.draw24(1234, 7, 3, 0, 20 + j) for j in range(4)] == [int(v >> 8) for v in blk]


def test_params_match_reference_constants(oracle_mod):
    P = oracle_mod.params(0.5, 1.0)
    # src/cuda/aco_cuda.cu:209-242 with rho=0.5, tau0=1
    assert P["q_evap_delta"] == 13
    assert P["q_tau0"] == 170
    assert abs(P["log_tau_step"] - 0.0541785) < 1e-6


def test_weight_tables(oracle_mod):
    O = oracle_mod
    A, lut, thr = O.tables(1.0, 2.0)
    assert A[0] == 0 and np.all(np.diff(A) >= 0) and A[255] == 319
    assert lut[0] == 1 << 23 and lut[255] == 0 and np.all(np.diff(lut[:255].astype(np.int64)) < 0)
    assert lut[16] == 1 << 22  # one octave per 16 levels
    finite = thr[np.isfinite(thr)]
    assert np.all(np.diff(finite) > 0)
    # beta = 2: L(d^2) counts 1/16-octave steps of d^2
    assert O.lib().orc_level(np.float32(1.0), thr.ctypes.data, len(thr)) == 0
    assert O.lib().orc_level(np.float32(2.0), thr.ctypes.data, len(thr)) == 16
    assert O.lib().orc_level(np.float32(4.0), thr.ctypes.data, len(thr)) == 32


def test_knn_order_and_exclusions(oracle_mod):
    O = oracle_mod
    inst = I.uniform_instance(150, 3, 11)
    k = 32
    cand = O.knn(inst.x, inst.y, k).reshape(-1, k)
    x, y = inst.x.astype(np.float64), inst.y.astype(np.float64)
    for i in range(inst.n + 1):
        row = cand[i]
        assert 0 not in row and i not in row and len(set(row)) == k
        d2 = (x[row] - x[i]) ** 2 + (y[row] - y[i]) ** 2
        keys = list(zip(d2, row))
        assert keys == sorted(keys)
        others = np.array([j for j in range(1, inst.n + 1) if j != i and j not in row])
        od2 = (x[others] - x[i]) ** 2 + (y[others] - y[i]) ** 2
        assert (od2.min(), 0) >= (d2[-1], 0) or od2.min() >= d2[-1]


def test_knn_small_n_pads_with_zero(oracle_mod):
    inst = I.uniform_instance(5, 2, 3)
    cand = oracle_mod.knn(inst.x, inst.y, 5).reshape(-1, 5)
    assert sorted(cand[0]) == [1, 2, 3, 4, 5]  # depot row: every customer
    for i in range(1, 6):
        assert cand[i][-1] == 0 and sorted(cand[i][:4]) == sorted(set(range(1, 6)) - {i})


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_golden(oracle_mod, path):
    O = oracle_mod
    g = np.load(path)
    K, cap, k = int(g["K"]), int(g["cap"]), int(g["k"])
    seed, epoch = int(g["seed"]), int(g["epoch"])
    x, y = g["x"], g["y"]
    A, lut, thr = O.tables(1.0, 2.0)
    # the oracle's own tables reproduce the fixture's inputs
    assert np.array_equal(O.knn(x, y, k), g["cand"])
    assert np.array_equal(O.levels(x, y, g["cand"], k, thr), g["lvl"])
    assert np.array_equal(O.weights(len(x) - 1, k, g["cand"], g["lvl"], g["tau"], A, lut), g["w"])
    for ant in range(g["costs"].size):
        feas, nodes, lens, cost, steps, used = O.construct_ant(
            x, y, None, K, cap, k, g["cand"], g["w"], seed, epoch, ant)
        exp_lens = g["lens"][ant]
        assert np.array_equal(lens, exp_lens), ant
        assert np.array_equal(nodes, g["nodes"][ant][: exp_lens.sum()]), ant
        assert cost == g["costs"][ant]
        assert used == g["draws_used"][ant]
        assert feas and steps == len(x) - 1 + K


def _ref_cases():
    return [
        (I.uniform_instance(40, 2, 901).unit_twin(), 32, 7, 0),
        (I.uniform_instance(5, 2, 902).unit_twin(), 5, 8, 1),       # n <= k: padded rows
        (I.uniform_instance(30, 1, 903).unit_twin(), 16, 9, 2),      # one vehicle
        (I.clustered_instance(400, 7, 904).unit_twin(), 32, 10, 5),  # duplicates likely
        (I.uniform_instance(250, 12, 905).unit_twin(), 8, 11, 4),    # short lists
    ]


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle",
                                                    "_ref", "libseqref.so")),
                    reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("case", range(5))
def test_oracle_matches_reference_harness(oracle_mod, case):
    O = oracle_mod
    inst, k, seed, epoch = _ref_cases()[case]
    n, K, cap = inst.n, inst.vehicles, inst.capacity
    k = min(k, n)
    A, lut, thr = O.tables(1.0, 2.0)
    cand = O.knn(inst.x, inst.y, k)
    lvl = O.levels(inst.x, inst.y, cand, k, thr)
    rs = np.random.RandomState(case)
    tau = rs.randint(0, 256, size=(n + 1) ** 2).astype(np.uint8)
    w = O.weights(n, k, cand, lvl, tau, A, lut)
    for ant in range(12):
        feas, nodes, lens, cost, steps, used = O.construct_ant(
            inst.x, inst.y, None, K, cap, k, cand, w, seed, epoch, ant)
        rn, rl, rc, ru = O.ref_construct_ant(inst.x, inst.y, K, cap, k, cand, w,
                                             O.draws(seed, epoch, ant, 0, n + K + 1))
        assert np.array_equal(nodes, rn) and np.array_equal(lens, rl)
        assert cost == rc and used == ru
        assert O.ref_validate(n, K, nodes, lens)
        assert O.route_cost(inst.x, inst.y, nodes, lens) == O.ref_cost(inst.x, inst.y, nodes, lens)


def test_demand_extension_reduces_to_unit(oracle_mod):
    O = oracle_mod
    inst = I.uniform_instance(120, 4, 71).unit_twin()
    k = 32
    A, lut, thr = O.tables()
    cand = O.knn(inst.x, inst.y, k)
    lvl = O.levels(inst.x, inst.y, cand, k, thr)
    tau = np.random.RandomState(2).randint(0, 256, size=(inst.n + 1) ** 2).astype(np.uint8)
    w = O.weights(inst.n, k, cand, lvl, tau, A, lut)
    for ant in range(8):
        a = O.construct_ant(inst.x, inst.y, None, 4, inst.capacity, k, cand, w, 3, 1, ant)
        b = O.construct_ant(inst.x, inst.y, inst.demand, 4, inst.capacity, k, cand, w, 3, 1, ant)
        assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
        assert a[3] == b[3] and a[5] == b[5]


def test_demand_routes_respect_capacity(oracle_mod):
    O = oracle_mod
    inst = I.uniform_instance(200, 5, 72, demand_max=100)
    k = 32
    A, lut, thr = O.tables()
    cand = O.knn(inst.x, inst.y, k)
    lvl = O.levels(inst.x, inst.y, cand, k, thr)
    tau = np.full((inst.n + 1) ** 2, 170, np.uint8)
    w = O.weights(inst.n, k, cand, lvl, tau, A, lut)
    nfeas = 0
    for ant in range(16):
        feas, nodes, lens, cost, steps, used = O.construct_ant(
            inst.x, inst.y, inst.demand, inst.vehicles, inst.capacity, k, cand, w, 5, 0, ant)
        off = 0
        seen = set()
        for ln in lens:
            r = nodes[off:off + ln]
            assert r[0] == 0 and r[-1] == 0 and 0 not in r[1:-1]
            assert inst.demand[r].sum() <= inst.capacity
            seen.update(int(v) for v in r[1:-1])
            off += ln
        assert feas == (len(seen) == inst.n)
        nfeas += feas
    assert nfeas > 0


def test_evaporate_exact(oracle_mod):
    tau = np.arange(256, dtype=np.uint8).repeat(3)
    for delta, qmin in [(13, 0), (1, 5), (200, 100), (13, 250)]:
        out = oracle_mod.evaporate(tau, delta, qmin)
        q = tau.astype(np.int32)
        exp = np.where(q > qmin + delta, q - delta, qmin).astype(np.uint8)
        assert np.array_equal(out, exp)


def test_deposit_touches_route_arcs_only(oracle_mod):
    O = oracle_mod
    P = O.params()
    n = 9
    tau = np.full((n + 1) ** 2, 100, np.uint8)
    nodes = np.array([0, 3, 4, 0, 0, 0, 5, 0, 0, 1, 2, 6, 7, 8, 9, 0], np.int32)
    lens = np.array([4, 2, 3, 7], np.int32)
    out = O.deposit(tau, n, nodes, lens, 50.0 / 1000.0 * 30, P["log_tau_min"], P["log_tau_step"])
    changed = set(map(tuple, np.argwhere(out.reshape(n + 1, n + 1) != 100)))
    arcs = set()
    off = 0
    for ln in lens:
        r = nodes[off:off + ln]
        for a, b in zip(r[:-1], r[1:]):
            arcs |= {(a, b), (b, a)}
        off += ln
    assert changed <= arcs and len(changed) > 0
    assert np.all(out >= tau)


def test_cuda_ref_depot_rule_serves_everyone(oracle_mod):
    """Reference-CUDA depot rule in the oracle: every customer served once,
    and with roomy capacity the routes differ from the sequential rule's."""
    import ctypes
    O = oracle_mod
    base = I.uniform_instance(150, 4, 905).unit_twin()
    inst = I.Instance("roomy", base.x, base.y, base.demand, 4, 80)
    n, K, k = inst.n, 4, 16
    A, lut, thr = O.tables()
    P = O.params()
    cand = O.knn(inst.x, inst.y, k)
    lvl = O.levels(inst.x, inst.y, cand, k, thr)
    tau = np.full((n + 1) ** 2, P["q_tau0"], np.uint8)
    w = O.weights(n, k, cand, lvl, tau, A, lut)
    d2 = ((inst.x - inst.x[0]) ** 2 + (inst.y - inst.y[0]) ** 2).astype(np.float32)
    lvl0 = np.array([O.lib().orc_level(float(v), thr.ctypes.data_as(ctypes.c_void_p), len(thr))
                     for v in d2], np.uint16)
    e_dep = int(round(16.0 * (1.0 - np.float64(np.float32(np.log(np.float32(1e-4)))) / np.log(2.0))))
    rdep = O.depot_rel(n, k, cand, lvl, tau, A, lvl0, e_dep)
    differs = 0
    for a in range(24):
        f, nodes, lens, cost, steps, used = O.construct_ant(
            inst.x, inst.y, None, K, inst.capacity, k, cand, w, 5, 0, a, rule=1, rdep=rdep,
            lut=lut)
        assert f and sorted(nodes[nodes > 0]) == list(range(1, n + 1))
        assert all(nodes[np.cumsum(lens) - 1] == 0) and lens.sum() == n + 2 * K
        f0, n0, l0, *_ = O.construct_ant(inst.x, inst.y, None, K, inst.capacity, k, cand, w,
                                         5, 0, a)
        differs += int(not np.array_equal(lens, l0) or not np.array_equal(nodes, n0))
    assert differs > 0


def _seq_update_loops(tau, n, solutions, rho, tau_min, tau_max, reset, tau0):
    """The reference's update written as its scalar loops
    (src/seq/aco_sequential.c:829-886), for small n."""
    t = [list(map(float, tau[i * (n + 1):(i + 1) * (n + 1)])) for i in range(n + 1)]
    for i in range(n + 1):
        for j in range(n + 1):
            if i != j:
                t[i][j] *= (1.0 - rho)
    for nodes, lens, d in solutions:
        e = 0
        for ln in lens:
            for q in range(ln - 1):
                u, v = int(nodes[e + q]), int(nodes[e + q + 1])
                t[u][v] += d
                t[v][u] += d
            e += ln
    for i in range(n + 1):
        for j in range(n + 1):
            if i == j:
                continue
            if t[i][j] < tau_min:
                t[i][j] = tau_min
            elif t[i][j] > tau_max:
                t[i][j] = tau_max
    if reset:
        for i in range(n + 1):
            for j in range(n + 1):
                if i != j:
                    t[i][j] = 0.5 * t[i][j] + 0.5 * tau0
    return np.array(t, np.float64).ravel()


@pytest.mark.parametrize("reset", [False, True])
def test_seq_update_restatement_equals_scalar_loops(oracle_mod, reset):
    n = 20
    rs = np.random.RandomState(3)
    tau = rs.uniform(0.001, 0.05, size=(n + 1) ** 2)
    it = (np.array([0, 3, 7, 0, 0, 0, 1, 2, 4, 5, 6, 8, 9, 10, 0], np.int32),
          np.array([4, 2, 9], np.int32), 0.013)
    gb = (np.array([0, 7, 3, 1, 0, 0, 2, 4, 5, 0, 0, 6, 8, 9, 10, 0], np.int32),
          np.array([5, 5, 6], np.int32), 0.021)
    got = oracle_mod.seq_pheromone_update(tau, n, it[0], it[1], it[2], gb[0], gb[1], gb[2],
                                          0.1, 0.004, 0.04, reset, 1.0)
    ref = _seq_update_loops(tau, n, [it, gb], 0.1, 0.004, 0.04, reset, 1.0)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
