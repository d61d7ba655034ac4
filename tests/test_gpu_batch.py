"""GPU tests of the batched solver: every instance of a batch gives exactly
what the single-instance solver gives with seed + i, whatever launch shape
(lanes per ant, ants per block, queue order) runs it."""
import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu


def mixed_instances():
    out = []
    for i, (n, K, dm) in enumerate([(20, 2, 30), (57, 3, 100), (140, 4, 100), (301, 6, 50),
                                    (96, 2, 1), (233, 5, 100), (17, 3, 100), (480, 9, 100)]):
        inst = I.uniform_instance(n, K, 950 + i, demand_max=max(dm, 1))
        out.append(inst.unit_twin() if dm == 1 else inst)
    out.append(I.clustered_instance(180, 4, 960))
    return out


def plain(inst, seed, ants, k, epochs, stagnation=0):
    with _native.Context(0) as ctx:
        ctx.setup_instance(inst, ants=ants, cand_k=k, seed=seed, fixed_epochs=epochs,
                           stagnation_epochs=stagnation)
        st = ctx.run(epochs)
        nodes, lens, cost = ctx.best()
        return nodes, lens, cost, st.epochs


@pytest.fixture(scope="module")
def reference_runs():
    insts = mixed_instances()
    return insts, [plain(inst, 500 + i, 16, 16, 12) for i, inst in enumerate(insts)]


@pytest.mark.parametrize("tuning", [(32, 16, 1), (32, 8, 0), (16, 16, 1), (16, 32, 0), (32, 32, 1)])
def test_batch_equals_single_instance_solver(reference_runs, tuning):
    insts, ref = reference_runs
    with _native.Batch(0) as b:
        b.setup(insts, ants=16, cand_k=16, seed=500, epochs=12)
        b.set_tuning(*tuning)
        b.solve()
        for i, (rn, rl, rc, re) in enumerate(ref):
            nodes, lens, cost, ep = b.best(i)
            assert ep == re == 12
            assert cost == rc, (i, cost, rc)
            assert np.array_equal(lens, rl) and np.array_equal(nodes, rn), i


def test_batch_stagnation_rule_matches():
    insts = mixed_instances()[:5]
    ref = [plain(inst, 77 + i, 16, 16, 200, stagnation=4) for i, inst in enumerate(insts)]
    with _native.Batch(0) as b:
        b.setup(insts, ants=16, cand_k=16, seed=77, epochs=200, stagnation_epochs=4)
        b.solve()
        for i, (rn, rl, rc, re) in enumerate(ref):
            nodes, lens, cost, ep = b.best(i)
            assert ep == re and cost == rc and np.array_equal(nodes, rn)


def test_autotune_keeps_results():
    insts = I.batched_instances(24, seed0=31000)
    with _native.Batch(0) as b:
        b.setup(insts, ants=32, cand_k=16, seed=9, epochs=6)
        chosen, ms = b.autotune(trial_epochs=2)
        assert len(ms) >= 6 and (ms > 0).sum() >= 6
        b.solve()
        c1, e1, s1 = b.costs()
        b.set_tuning(32, 16, 0)
        b.solve()
        c2, e2, s2 = b.costs()
        assert np.array_equal(c1, c2) and np.array_equal(e1, e2) and np.array_equal(s1, s2)
        assert np.all(e1 == 6) and np.all(np.isfinite(c1) | (c1 > 1e300))
    for i in (0, 7, 23):
        assert plain(insts[i], 9 + i, 32, 16, 6)[2] == c1[i]


@pytest.mark.parametrize("k", [20, 32, 12])
def test_set_cand_k_equals_single_instance_solver(k):
    """Candidate lists rebuilt in place with another length give what the
    single-instance solver gives at that length."""
    insts = I.batched_instances(10, seed0=31500)
    with _native.Batch(0) as b:
        b.setup(insts, ants=16, cand_k=16, seed=40, epochs=8)
        b.set_cand_k(k)
        assert b.cand_k() == k
        if k > 16:
            assert b.tuning()[0] == 32  # 16 lanes cannot hold the list
        b.solve()
        for i in (0, 3, 9):
            rn, rl, rc, re = plain(insts[i], 40 + i, 16, k, 8)
            nodes, lens, cost, ep = b.best(i)
            assert cost == rc and np.array_equal(nodes, rn) and np.array_equal(lens, rl)


def test_autotune_chooses_candidate_length():
    insts = I.batched_instances(24, seed0=31000)
    with _native.Batch(0) as b:
        b.setup(insts, ants=32, cand_k=16, seed=9, epochs=6)
        k, shape, per, ms = b.autotune_k(ks=(16, 20, 32), quality_tol=0.005, trial_epochs=2)
        assert b.cand_k() == k and b.tuning() == shape
        assert sorted(per) == [16, 20, 32] and all(v[0] > 0 for v in per.values())
        most = max(v[2] for v in per.values())
        best = min(v[1] for v in per.values() if v[2] == most)
        allowed = [kk for kk, v in per.items() if v[2] == most and v[1] <= best * 1.005]
        assert k == min(allowed, key=lambda kk: per[kk][0])
        assert len(ms) >= 3
        b.solve()
        c1, e1, _ = b.costs()
        assert np.all(e1 == 6)
    for i in (0, 7, 23):
        assert plain(insts[i], 9 + i, 32, k, 6)[2] == c1[i]


def test_setup_reuse_and_get_all(reference_runs):
    """One batch object solving a stream of batches: a smaller batch reuses
    the device buffers, a larger one reallocates them; every solve equals a
    fresh object's, and get_all returns what the per-instance getter does."""
    insts, ref = reference_runs
    small = insts[:3]
    large = insts + I.batched_instances(6, seed0=31500)
    with _native.Batch(0) as fresh:
        fresh.setup(large, ants=16, cand_k=16, seed=500, epochs=12)
        fresh.solve()
        want_large = [fresh.best(i) for i in range(len(large))]
    with _native.Batch(0) as b:
        for batch in (insts, small, insts, large):
            b.setup(batch, ants=16, cand_k=16, seed=500, epochs=12)
            b.solve()
            got = b.best_all()
            assert len(got) == len(batch)
            for i, (nodes, lens, cost) in enumerate(got):
                one = b.best(i)
                assert np.array_equal(nodes, one[0]) and np.array_equal(lens, one[1])
                assert cost == one[2]
                want = ref[i][:3] if batch is not large else want_large[i][:3]
                assert cost == want[2], (i, cost, want[2])
                assert np.array_equal(nodes, want[0]) and np.array_equal(lens, want[1])


def test_batch_with_an_unservable_instance():
    """An instance no ant can serve ends with no solution (infinite cost, no
    routes, pheromone untouched by the deposits) without disturbing the
    others, which equal the single-instance solver."""
    from tests.test_gpu_sharding import _unservable
    insts = [mixed_instances()[0], _unservable(), mixed_instances()[2]]
    want = [plain(insts[i], 40 + i, 16, 8, 10) for i in (0, 2)]
    with _native.Batch(0) as b:
        b.setup(insts, ants=16, cand_k=8, seed=40, epochs=10)
        b.solve()
        got = b.best_all()
        costs, epochs, steps = b.costs()
    assert got[1][2] == float("inf") and got[1][0].size == 0
    assert np.all(epochs == 10)
    for g, (rn, rl, rc, re) in zip((got[0], got[2]), want):
        assert g[2] == rc and np.array_equal(g[0], rn) and np.array_equal(g[1], rl)
