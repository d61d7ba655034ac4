"""GPU parity tests: the CUDA path through the C ABI against the oracle.

Bars: bit-exact candidate lists, eta levels, weights, routes, draw counts and
evaporated pheromone; FP64 route costs equal to the oracle's (same summation
order) and within 1e-9 relative of an independent FP64 recomputation;
deposited pheromone bit-exact against the reference's own CUDA kernels
(oracle/_ref/librefcuda.so) and within one level of the host-libm oracle.
"""
import ctypes as C
import os

import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFCUDA = os.path.join(ROOT, "oracle", "_ref", "librefcuda.so")
SEQREF = os.path.join(ROOT, "oracle", "_ref", "libseqref.so")


def smoke_instance():
    xs = np.array([50, 10, 20, 10, 20, 80, 90, 80, 90], np.float32)
    ys = np.array([50, 10, 10, 20, 20, 80, 80, 90, 90], np.float32)
    d = np.ones(9, np.int32)
    d[0] = 0
    return I.Instance("smoke", xs, ys, d, 2, 5)


CASES = {
    "smoke": (smoke_instance, 8, 16),
    "u200_unit": (lambda: I.uniform_instance(200, 4, 601).unit_twin(), 32, 48),
    "small_c1": (I.workload_small, 20, 128),
    "u300_demand": (lambda: I.uniform_instance(300, 5, 602), 20, 40),
    "n1000_c2": (I.workload_n1000, 32, 256),
    "n1000_unit": (lambda: I.workload_n1000().unit_twin(), 32, 96),
    "c2000_demand": (lambda: I.clustered_instance(2000, 16, 603), 32, 64),
    # n >= 2048: visited bitmap in shared memory, rows read from global memory
    "u3000_demand": (lambda: I.uniform_instance(3000, 24, 604), 32, 32),
    # K > 4096 routes of one or two customers: the deposit's unstaged path
    "many_vehicles": (lambda: I.Instance("mv", *_many_vehicles()), 8, 8),
    # the clustered n=2000 workload as benched: 1024 ants, 7 ants per block,
    # packed levels in shared memory
    "c3_bench": (I.workload_clustered2000, 32, 1024),
    # n=16000: visited bitmap in shared memory, rows from global memory, in
    # the reference's published CUDA size range
    "u16000_unit": (lambda: I.uniform_instance(16000, 16, 660).unit_twin(), 32, 16),
}
# Cases checked on every STRIDE-th ant only (the oracle is sequential).
STRIDE = {"c3_bench": 8}


def _many_vehicles():
    base = I.uniform_instance(5000, 4200, 605).unit_twin()
    return base.x, base.y, base.demand, 4200, 2


def make_ctx(inst, k, m, seed=1234, **kw):
    ctx = _native.Context(0)
    ctx.setup_instance(inst, ants=m, cand_k=k, seed=seed, **kw)
    return ctx


def random_tau(n, seed, mode="random"):
    rs = np.random.RandomState(seed)
    if mode == "random":
        return rs.randint(0, 256, size=(n + 1) ** 2).astype(np.uint8)
    t = np.full((n + 1) ** 2, 170, np.uint8)
    idx = rs.randint(0, t.size, size=t.size // 10)
    t[idx] = rs.randint(0, 256, size=idx.size).astype(np.uint8)
    return t


def fp64_cost(inst, nodes, lens):
    x = inst.x.astype(np.float64)
    y = inst.y.astype(np.float64)
    tot, off = 0.0, 0
    for ln in lens:
        r = nodes[off:off + ln]
        tot += float(np.sum(np.hypot(x[r[1:]] - x[r[:-1]], y[r[1:]] - y[r[:-1]])))
        off += ln
    return tot


@pytest.mark.parametrize("name", ["smoke", "u200_unit", "u300_demand", "n1000_c2", "c2000_demand"])
def test_candidates_levels_tables(oracle_mod, name):
    O = oracle_mod
    factory, k, m = CASES[name]
    inst = factory()
    with make_ctx(inst, k, 8) as ctx:
        A, lut, thr = ctx.tables()
        oA, olut, othr = O.tables(1.0, 2.0)
        assert np.array_equal(A, oA) and np.array_equal(lut, olut)
        assert np.array_equal(thr.view(np.uint32), othr.view(np.uint32))
        cand, lvl = ctx.candidates()
        kk = ctx.k
        ocand = O.knn(inst.x, inst.y, kk)
        assert np.array_equal(cand, ocand)
        assert np.array_equal(lvl, O.levels(inst.x, inst.y, ocand, kk, othr))


@pytest.mark.parametrize("name", ["smoke", "small_c1", "u300_demand", "n1000_c2", "c2000_demand"])
def test_fallback_tier_lists(oracle_mod, name):
    """The fallback's neighbour lists: ranks k+1 .. k+64 of the oracle's
    nearest-neighbour order (0 where fewer customers exist)."""
    factory, k, m = CASES[name]
    inst = factory()
    with make_ctx(inst, k, 8) as ctx:
        kk = ctx.k
        full = oracle_mod.knn(inst.x, inst.y, kk + 64).reshape(inst.n + 1, kk + 64)
        assert np.array_equal(ctx.tier().reshape(inst.n + 1, 64), full[:, kk:].astype(np.uint16))


def test_fallback_second_tier_lists(oracle_mod):
    """The second tier of a large instance (n >= 1500): ranks k+65 .. k+256
    of the oracle's nearest-neighbour order; smaller instances have none."""
    inst = I.uniform_instance(4500, 12, 7801)
    with make_ctx(inst, 32, 8) as ctx:
        full = oracle_mod.knn(inst.x, inst.y, 32 + 256).reshape(inst.n + 1, 32 + 256)
        assert np.array_equal(ctx.tier().reshape(inst.n + 1, 64), full[:, 32:96].astype(np.uint16))
        assert np.array_equal(ctx.tier2().reshape(inst.n + 1, 192), full[:, 96:].astype(np.uint16))
    c2 = CASES["c2000_demand"][0]()  # clustered n=2000: the register bitmap of two words
    with make_ctx(c2, 32, 8) as ctx:
        full = oracle_mod.knn(c2.x, c2.y, 32 + 256).reshape(c2.n + 1, 32 + 256)
        assert np.array_equal(ctx.tier2().reshape(c2.n + 1, 192), full[:, 96:].astype(np.uint16))
    with make_ctx(CASES["n1000_c2"][0](), 32, 8) as ctx:
        with pytest.raises(_native.AcoError):
            ctx.tier2()


@pytest.mark.parametrize("name", ["u200_unit", "u300_demand", "n1000_c2"])
@pytest.mark.parametrize("mode", ["random", "mostly_init"])
def test_weights(oracle_mod, name, mode):
    O = oracle_mod
    factory, k, m = CASES[name]
    inst = factory()
    with make_ctx(inst, k, 8) as ctx:
        tau = random_tau(inst.n, 5, mode)
        ctx.set_tau(tau)
        cand, lvl = ctx.candidates()
        A, lut, _ = O.tables()
        assert np.array_equal(ctx.weights(), O.weights(inst.n, ctx.k, cand, lvl, tau, A, lut))


def check_construct(O, inst, ctx, seed, epoch, tau, ants=None):
    n, K = inst.n, inst.vehicles
    cand, lvl = ctx.candidates()
    A, lut, _ = O.tables()
    w = O.weights(n, ctx.k, cand, lvl, tau, A, lut)
    nodes, lens, cost, feas, steps, draws = ctx.ants()
    demand = None if inst.is_unit_demand() else inst.demand
    ants = range(ctx.m) if ants is None else ants
    for a in ants:
        of, on, ol, oc, osteps, oused = O.construct_ant(
            inst.x, inst.y, demand, K, inst.capacity, ctx.k, cand, w, seed, epoch, a)
        assert np.array_equal(lens[a], ol), f"ant {a}: lens {lens[a]} vs {ol}"
        assert np.array_equal(nodes[a][: ol.sum()], on), f"ant {a}: routes differ"
        assert cost[a] == oc, f"ant {a}: cost {cost[a]!r} vs {oc!r}"
        assert bool(feas[a]) == of and steps[a] == osteps and draws[a] == oused
        ref = fp64_cost(inst, on, ol)
        assert abs(cost[a] - ref) <= 1e-9 * ref
    return nodes, lens, cost, feas


@pytest.mark.parametrize("name", ["smoke", "u200_unit", "small_c1", "u300_demand", "n1000_c2",
                                  "n1000_unit", "c2000_demand", "u3000_demand",
                                  "many_vehicles", "c3_bench", "u16000_unit"])
def test_construct_matches_oracle(oracle_mod, name):
    factory, k, m = CASES[name]
    inst = factory()
    ants = range(0, m, STRIDE.get(name, 1))
    with make_ctx(inst, k, m, seed=4321) as ctx:
        for epoch, mode in [(0, None), (3, "random"), (9, "mostly_init")]:
            tau = ctx.tau() if mode is None else random_tau(inst.n, epoch, mode)
            ctx.set_tau(tau)
            ctx.construct(epoch)
            check_construct(oracle_mod, inst, ctx, 4321, epoch, tau, ants=ants)


def test_benched_shapes_take_the_tested_plans():
    """The launch shapes the parity cases above stand for: the clustered
    n=2000 workload as benched runs 7 ants per block on packed levels in
    shared memory, n=16000 reads rows from global memory with the visited
    bitmap in shared memory."""
    with make_ctx(I.workload_clustered2000(), 32, 1024) as ctx:
        plan = ctx.plan()
        assert plan["wpb"] == 7 and plan["layout"] == _native.LAYOUT_SMEM_PACKED
    with make_ctx(CASES["u16000_unit"][0](), 32, 16) as ctx:
        plan = ctx.plan()
        assert plan["layout"] == _native.LAYOUT_GLOBAL and plan["vreg"] == 0


@pytest.mark.parametrize("layout", [_native.LAYOUT_SMEM_WEIGHTS, _native.LAYOUT_SMEM_PACKED,
                                    _native.LAYOUT_GLOBAL])
@pytest.mark.parametrize("name", ["u200_unit", "u300_demand"])
def test_construct_layouts_agree(oracle_mod, name, layout):
    factory, k, m = CASES[name]
    inst = factory()
    with make_ctx(inst, k, m, seed=99) as ctx:
        tau = random_tau(inst.n, 21, "mostly_init")
        ctx.set_tau(tau)
        ctx.construct(2, layout)
        check_construct(oracle_mod, inst, ctx, 99, 2, tau)


def test_construct_layouts_large(oracle_mod):
    factory, k, m = CASES["c2000_demand"]
    inst = factory()
    with make_ctx(inst, k, m, seed=7) as ctx:
        tau = random_tau(inst.n, 3, "mostly_init")
        ctx.set_tau(tau)
        for layout in (_native.LAYOUT_SMEM_PACKED, _native.LAYOUT_GLOBAL):
            ctx.construct(1, layout)
            check_construct(oracle_mod, inst, ctx, 7, 1, tau, ants=range(0, m, 4))


@pytest.mark.skipif(not os.path.exists(SEQREF), reason="oracle/_ref not built")
def test_construct_matches_reference_seq_code(oracle_mod):
    """GPU routes equal the reference's own build_ant_solution on the same
    candidate lists, weights and recorded draws."""
    O = oracle_mod
    inst = I.workload_n1000().unit_twin()
    with make_ctx(inst, 32, 64, seed=2024) as ctx:
        tau = random_tau(inst.n, 8)
        ctx.set_tau(tau)
        ctx.construct(5)
        nodes, lens, cost, feas, steps, draws = ctx.ants()
        cand, lvl = ctx.candidates()
        A, lut, _ = O.tables()
        w = O.weights(inst.n, 32, cand, lvl, tau, A, lut)
        for a in range(64):
            rn, rl, rc, ru = O.ref_construct_ant(inst.x, inst.y, inst.vehicles, inst.capacity,
                                                 32, cand, w,
                                                 O.draws(2024, 5, a, 0, inst.n + inst.vehicles + 1))
            assert np.array_equal(lens[a], rl) and np.array_equal(nodes[a][: rl.sum()], rn)
            assert abs(cost[a] - rc) <= 1e-9 * rc and draws[a] == ru


def _compact_to_interleaved(nodes, lens):
    """Compact routes -> the reference's shared-depot step sequence."""
    seq = [0]
    off = 0
    for ln in lens:
        seq.extend(int(v) for v in nodes[off + 1: off + ln])
        off += ln
    return np.array(seq, np.int32)


def _compact_to_flat(nodes, lens, n):
    flat = np.zeros(len(lens) * (n + 1), np.int32)
    off = 0
    for v, ln in enumerate(lens):
        flat[v * (n + 1): v * (n + 1) + ln] = nodes[off: off + ln]
        off += ln
    return flat


@pytest.mark.parametrize("name", ["u200_unit", "n1000_c2", "many_vehicles"])
def test_evaporate_deposit(oracle_mod, name):
    O = oracle_mod
    factory, k, m = CASES[name]
    inst = factory()
    n = inst.n
    with make_ctx(inst, k, m, seed=5) as ctx:
        tau0 = random_tau(n, 44, "mostly_init")
        ctx.set_tau(tau0)
        ctx.construct(0)
        nodes, lens, cost, feas, _, _ = ctx.ants()
        best = int(np.argmin(np.where(feas > 0, cost, np.inf)))
        other = (best + 1) % ctx.m
        gn, gl = nodes[other][: lens[other].sum()], lens[other]
        di, dg = np.float32(0.3 * 100) / np.float32(cost[best]), np.float32(0.7 * 100) / np.float32(cost[other])
        ctx.set_tau(tau0)
        ctx.evaporate_deposit(best, float(di), gn, gl, float(dg))
        got = ctx.tau()
        P = O.params()
        evap = O.evaporate(tau0, P["q_evap_delta"])
        exp = O.deposit(evap, n, nodes[best][: lens[best].sum()], lens[best], float(di),
                        P["log_tau_min"], P["log_tau_step"])
        exp = O.deposit(exp, n, gn, gl, float(dg), P["log_tau_min"], P["log_tau_step"])
        arcs = np.zeros((n + 1, n + 1), bool)
        for nd, ln in ((nodes[best], lens[best]), (gn, gl)):
            off = 0
            for L in ln:
                r = nd[off: off + L]
                arcs[r[:-1], r[1:]] = True
                arcs[r[1:], r[:-1]] = True
                off += L
        arcs = arcs.ravel()
        assert np.array_equal(got[~arcs], evap[~arcs])          # evaporation: exact
        assert np.array_equal(got[~arcs], exp[~arcs])
        diff = np.abs(got[arcs].astype(int) - exp[arcs].astype(int))
        assert diff.max() <= 1 and (diff > 0).mean() < 0.02     # host libm vs device math


@pytest.mark.skipif(not os.path.exists(REFCUDA), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["u200_unit", "n1000_c2", "smoke"])
def test_kernels_match_reference_cuda(oracle_mod, name):
    """kNN order, evaporation and both deposits byte-for-byte against the
    reference's own kernels run on the same GPU."""
    import torch

    class CudaParams(C.Structure):
        _fields_ = [("n", C.c_int), ("K", C.c_int), ("m", C.c_int), ("cap", C.c_int),
                    ("cand_k", C.c_int), ("route_max_len", C.c_int),
                    ("alpha", C.c_float), ("beta", C.c_float), ("rho", C.c_float),
                    ("tau0", C.c_float), ("Q", C.c_float), ("tau_min", C.c_float),
                    ("tau_max", C.c_float), ("log_tau_min", C.c_float),
                    ("log_tau_step", C.c_float), ("q_tau_min", C.c_uint8),
                    ("q_tau_max", C.c_uint8), ("q_evap_delta", C.c_uint8),
                    ("visited_l1_words", C.c_int), ("visited_l2_words", C.c_int),
                    ("visited_row_stride", C.c_size_t), ("depot_close_weight", C.c_float)]

    R = C.CDLL(REFCUDA)
    R.refcuda_params_size.restype = C.c_int
    assert R.refcuda_params_size() == C.sizeof(CudaParams)
    for fn in ("refcuda_evaporate", "refcuda_build_candidates", "refcuda_deposit_solution",
               "refcuda_deposit_flat"):
        getattr(R, fn).restype = C.c_int
    R.refcuda_evaporate.argtypes = [C.c_void_p, C.c_int, C.c_uint8, C.c_uint8]
    R.refcuda_build_candidates.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    R.refcuda_deposit_solution.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                           C.c_int, C.c_void_p]
    R.refcuda_deposit_flat.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                       C.c_void_p]
    O = oracle_mod
    factory, k, m = CASES[name]
    inst = factory()
    n, K = inst.n, inst.vehicles
    P = O.params()
    with make_ctx(inst, k, m, seed=31) as ctx:
        kk = ctx.k
        prm = CudaParams(n=n, K=K, m=1, cap=inst.capacity, cand_k=kk, route_max_len=K * (n + 1),
                         alpha=1.0, beta=2.0, rho=0.5, tau0=1.0, Q=100.0, tau_min=1e-4,
                         tau_max=100.0, log_tau_min=P["log_tau_min"],
                         log_tau_step=P["log_tau_step"], q_tau_min=0, q_tau_max=255,
                         q_evap_delta=P["q_evap_delta"], visited_l1_words=(n + 64) // 64,
                         visited_l2_words=1, visited_row_stride=128, depot_close_weight=2.0)
        dev = torch.device("cuda", 0)
        xy = torch.tensor(np.stack([inst.x, inst.y], 1).ravel(), dtype=torch.float32, device=dev)
        ridx = torch.zeros((n + 1) * kk, dtype=torch.int32, device=dev)
        reta = torch.zeros((n + 1) * kk, dtype=torch.float32, device=dev)
        assert R.refcuda_build_candidates(xy.data_ptr(), ridx.data_ptr(), reta.data_ptr(),
                                          C.byref(prm)) == 0
        cand, _ = ctx.candidates()
        assert np.array_equal(cand, ridx.cpu().numpy())

        tau0 = random_tau(n, 12, "mostly_init")
        ctx.set_tau(tau0)
        ctx.construct(1)
        nodes, lens, cost, feas, _, _ = ctx.ants()
        best = int(np.argmin(np.where(feas > 0, cost, np.inf)))
        other = (best + 3) % ctx.m
        bn, bl = nodes[best][: lens[best].sum()], lens[best]
        gn, gl = nodes[other][: lens[other].sum()], lens[other]
        di = float(np.float32(30.0) / np.float32(cost[best]))
        dg = float(np.float32(70.0) / np.float32(cost[other]))
        ctx.set_tau(tau0)
        ctx.evaporate_deposit(best, di, gn, gl, dg)
        got = ctx.tau()

        alloc = ((n + 1) ** 2 + 3) & ~3
        rt = torch.zeros(alloc, dtype=torch.uint8, device=dev)
        rt[: tau0.size] = torch.from_numpy(tau0).to(dev)
        assert R.refcuda_evaporate(rt.data_ptr(), n, P["q_evap_delta"], 0) == 0
        steps = torch.from_numpy(_compact_to_interleaved(bn, bl)).to(dev)
        rlens = torch.from_numpy(bl.astype(np.int32)).to(dev)
        assert R.refcuda_deposit_solution(rt.data_ptr(), steps.data_ptr(), rlens.data_ptr(),
                                          di, 0, C.byref(prm)) == 0
        flat = torch.from_numpy(_compact_to_flat(gn, gl, n)).to(dev)
        flens = torch.from_numpy(gl.astype(np.int32)).to(dev)
        assert R.refcuda_deposit_flat(rt.data_ptr(), flat.data_ptr(), flens.data_ptr(), dg,
                                      C.byref(prm)) == 0
        ref = rt.cpu().numpy()[: tau0.size]
        mask = np.ones(tau0.size, bool)
        if (bl == 2).sum() + (gl == 2).sum() >= 2:
            mask[0] = False  # the reference races on the depot loop cell
        assert np.array_equal(got[mask], ref[mask])


def test_epochs_follow_oracle(oracle_mod):
    """Several device epochs (graph-launched, device-side bookkeeping) against
    the oracle fed each epoch's starting pheromone."""
    O = oracle_mod
    inst = I.uniform_instance(150, 4, 611)
    n, K = inst.n, inst.vehicles
    m = 48
    P = O.params()
    A, lut, _ = O.tables()
    with make_ctx(inst, 20, m, seed=77, stagnation_epochs=0) as ctx:
        cand, lvl = ctx.candidates()
        gbest = np.inf
        gnodes = glens = None
        since = 0
        for e in range(12):
            tau = ctx.tau()
            w = O.weights(n, ctx.k, cand, lvl, tau, A, lut)
            res = [O.construct_ant(inst.x, inst.y, inst.demand, K, inst.capacity, ctx.k, cand,
                                   w, 77, e, a) for a in range(m)]
            costs = np.array([r[3] if r[0] else np.inf for r in res])
            st = ctx.run(1)
            assert st.epochs == e + 1 and st.error == 0
            if not np.isfinite(costs).any():
                since += 1
                assert not st.found and st.iter_since_best == since
                continue
            b = int(np.argmin(costs))
            assert st.found and st.best_ant == b and st.iter_best == costs[b]
            if costs[b] < gbest:
                rel = (gbest - costs[b]) / gbest if np.isfinite(gbest) else 1.0
                since = 0 if (not np.isfinite(gbest) or (costs[b] < gbest - 1e-9 and rel + 1e-9 >= 1e-3)) else since + 1
                gbest = costs[b]
                gnodes, glens = res[b][1], res[b][2]
            else:
                since += 1
            assert st.global_best == gbest and st.iter_since_best == since
            assert st.dep_iter == np.float32(np.float32(0.3) * np.float32(100.0)) / np.float32(costs[b])
            bn, bl, bc = ctx.best()
            assert bc == gbest and np.array_equal(bl, glens) and np.array_equal(bn, gnodes)
            got = ctx.tau()
            evap = O.evaporate(tau, P["q_evap_delta"])
            exp = O.deposit(evap, n, res[b][1], res[b][2], float(st.dep_iter),
                            P["log_tau_min"], P["log_tau_step"])
            exp = O.deposit(exp, n, gnodes, glens, float(st.dep_global), P["log_tau_min"],
                            P["log_tau_step"])
            d = np.abs(got.astype(int) - exp.astype(int))
            assert d.max() <= 1 and (d > 0).sum() <= 4


def test_stop_rules_and_determinism():
    inst = I.uniform_instance(120, 3, 612)
    with make_ctx(inst, 16, 32, seed=3, stagnation_epochs=4) as ctx:
        st = ctx.run(500)
        assert st.stopped and st.stop_reason & 1 and st.iter_since_best >= 4
        assert st.epochs < 500
        t1, b1 = ctx.tau(), ctx.best()
    with make_ctx(inst, 16, 32, seed=3, stagnation_epochs=4) as ctx:
        st2 = ctx.run(500)
        assert st2.epochs == st.epochs and st2.global_best == st.global_best
        assert np.array_equal(ctx.tau(), t1) and np.array_equal(ctx.best()[0], b1[0])
    with make_ctx(inst, 16, 32, seed=3, fixed_epochs=7) as ctx:
        st = ctx.run(100)
        assert st.epochs == 7 and st.stop_reason & 2
    with make_ctx(inst, 16, 32, seed=3) as ctx:
        st = ctx.run(21)  # chunked graph launches plus single epochs
        assert st.epochs == 21 and not st.stopped
        st = ctx.run(5)
        assert st.epochs == 26


def test_setup_reuse_matches_fresh_contexts():
    """A context set up again with the same sizes keeps its buffers and, when
    the captured arguments match, its epoch graphs; every solve must equal a
    fresh context's (seed, instance and parameters changed in between)."""
    a = I.uniform_instance(180, 4, 620)
    b = I.uniform_instance(180, 4, 621)  # same sizes, other coordinates and demands
    runs = [(a, 5, 0.5), (a, 6, 0.5), (b, 6, 0.5), (a, 7, 0.3), (a, 5, 0.5)]
    with make_ctx(a, 24, 40, seed=5) as reused:
        for inst, seed, rho in runs:
            reused.setup_instance(inst, ants=40, cand_k=24, seed=seed, rho=rho)
            st = reused.run(21)
            with make_ctx(inst, 24, 40, seed=seed, rho=rho) as fresh:
                sf = fresh.run(21)
                assert (st.epochs, st.global_best, st.total_steps, st.iter_since_best) == \
                    (sf.epochs, sf.global_best, sf.total_steps, sf.iter_since_best)
                assert np.array_equal(reused.tau(), fresh.tau())
                bn, bl, bc = reused.best()
                fn, fl, fc = fresh.best()
                assert bc == fc and np.array_equal(bn, fn) and np.array_equal(bl, fl)


# staged weights, packed levels, global rows; n=8000 with the bitmap in shared memory
@pytest.mark.parametrize("n", [400, 1500, 3000, 8000])
def test_recorded_draws_match_reference_seq_code(oracle_mod, n):
    """The harness of the parity contract: the GPU construction and the
    reference's own build_ant_solution (src/seq/aco_sequential.c:616-681,
    compiled from its sources) fed the same candidate lists, weights and an
    arbitrary recorded stream of draws give the same routes."""
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    O = oracle_mod
    inst = I.uniform_instance(n, 6 + n // 500, 640 + n).unit_twin()
    m, k = 16, 32
    rs = np.random.RandomState(n)
    draws = rs.randint(0, 1 << 24, size=(m, inst.n + inst.vehicles + 8)).astype(np.uint32)
    with make_ctx(inst, k, m, seed=1) as ctx:
        ctx.set_tau(random_tau(inst.n, 9 + n))
        ctx.construct_with_draws(draws)
        nodes, lens, cost, feas, steps, used = ctx.ants()
        cand, lvl = ctx.candidates()
        A, lut, _ = O.tables()
        w = O.weights(inst.n, k, cand, lvl, ctx.tau(), A, lut)
        refs = O.ref_construct_ants(inst.x, inst.y, inst.vehicles, inst.capacity, k, cand, w,
                                    draws)
        for a, (rn, rl, rc, ru) in enumerate(refs):
            assert np.array_equal(lens[a], rl) and np.array_equal(nodes[a][: rl.sum()], rn)
            assert abs(cost[a] - rc) <= 1e-9 * rc and used[a] == ru
        # Philox draws recorded and replayed give the Philox run's routes
        ctx.construct(3)
        n1, l1, *_ = ctx.ants()
        rec = np.stack([O.draws(1, 3, a, 0, inst.n + inst.vehicles + 8) for a in range(m)])
        ctx.construct_with_draws(rec)
        n2, l2, *_ = ctx.ants()
        assert np.array_equal(n1, n2) and np.array_equal(l1, l2)
