"""Learned heuristic prior on the GPU against the FP64 oracle
(oracle/prior_oracle.py): features, elite examples, the tensor-core forward
pass, the gradient of the training loss, the Adam step, the learned levels
and their use by the exact construction path."""
import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu

K_CAND = 32


def _instances():
    return [I.uniform_instance(40, 2, 811, demand_max=20),
            I.uniform_instance(120, 3, 812),
            I.clustered_instance(300, 5, 813),
            I.uniform_instance(200, 4, 814, demand_max=1),
            I.clustered_instance(90, 2, 815)]


@pytest.fixture(scope="module")
def dataset(native):
    insts = _instances()
    sols = []
    for j, inst in enumerate(insts):
        with native.Context(0) as c:
            c.setup_instance(inst, ants=32, cand_k=16, seed=70 + j)
            c.run(25)
            nodes, lens, cost = c.best()
            assert np.isfinite(cost)
            sols.append((nodes, lens))
    pr = native.Prior(0, seed=1234)
    cnt = pr.set_dataset(insts, sols, cand_k=K_CAND)
    offs = np.cumsum([0] + [x.n + 1 for x in insts])
    yield insts, sols, pr, cnt, offs
    pr.close()


def _bits_to_f(bits):
    from oracle import prior_oracle as PO
    return PO.bf16_bits_to_float(bits)


def test_features_match_oracle(dataset, oracle_mod):
    from oracle import prior_oracle as PO
    insts, _, pr, _, offs = dataset
    for inst, off in zip(insts, offs):
        cand = oracle_mod.knn(inst.x, inst.y, min(K_CAND, inst.n))
        k = min(K_CAND, inst.n)
        F, kv = PO.features(inst.x, inst.y, inst.demand, inst.capacity, cand, k)
        bits, gkv, _ = pr.rows(int(off), inst.n + 1)
        assert np.array_equal(gkv.astype(np.int64), kv)
        got = _bits_to_f(bits)
        exp = PO.bf16(F)
        # FP32 on the device, FP64 here: equal after BF16 rounding, or one
        # BF16 step apart where the value sits on a rounding boundary
        diff = np.abs(got - exp)
        step = np.maximum(np.abs(exp), 1e-30) * 2.0 ** -7
        assert np.all(diff <= step * 1.01)
        assert (diff > 0).mean() < 0.01


def test_examples_follow_elite_routes(dataset, oracle_mod):
    insts, sols, pr, cnt, offs = dataset
    exp = []
    for inst, (nodes, lens), off in zip(insts, sols, offs):
        k = min(K_CAND, inst.n)
        cand = oracle_mod.knn(inst.x, inst.y, k).reshape(inst.n + 1, k)
        pos = 0
        for L in lens:
            r = nodes[pos:pos + L]
            pos += L
            pairs = []
            if L > 2:
                pairs.append((0, r[1]))
            for t in range(1, L - 2):
                pairs += [(r[t], r[t + 1]), (r[t + 1], r[t])]
            for a, b in pairs:
                hit = np.nonzero(cand[a] == b)[0]
                if len(hit):
                    exp.append((off + a, int(hit[0])))
    got = pr.examples()
    assert cnt == len(exp) == len(got) and cnt > 500
    assert [tuple(x) for x in got] == exp


def test_forward_matches_oracle(dataset):
    from oracle import prior_oracle as PO
    insts, _, pr, _, offs = dataset
    params = pr.params().astype(np.float64)
    rows = int(offs[-1])
    bits, kv, sc = pr.rows(0, rows, scores=True)
    X = _bits_to_f(bits)
    ref = PO.forward(params, X, kv.astype(np.int64), mimic=True)
    mask = np.arange(32)[None, :] < kv[:, None]
    err = np.abs(sc - ref)[mask]
    scale = np.abs(ref[mask]).max()
    assert err.max() <= 2e-3 * scale + 1e-4


@pytest.mark.parametrize("count", [1, 37, 512])
def test_gradient_matches_oracle(dataset, count):
    """Gradient check: tensor-core backward against the oracle's FP64
    backward (BF16 rounding at the device's points; the oracle's own
    gradient is pinned by finite differences in tests/test_prior_oracle.py)."""
    from oracle import prior_oracle as PO
    insts, _, pr, cnt, offs = dataset
    rs = np.random.RandomState(count)
    ids = rs.choice(cnt, count, replace=False).astype(np.int32)
    loss, g = pr.gradient(ids)
    params = pr.params().astype(np.float64)
    rows = int(offs[-1])
    bits, kv, _ = pr.rows(0, rows)
    X = _bits_to_f(bits)
    ex = pr.examples()[ids]
    ref_loss, ref = PO.loss_grad(params, X, kv.astype(np.int64), ex, mimic=True)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert rel < 2e-3, rel
    # and against the exact FP64 model (no BF16 rounding)
    _, exact = PO.loss_grad(params, X, kv.astype(np.int64), ex, mimic=False)
    assert np.linalg.norm(g - exact) / np.linalg.norm(exact) < 5e-2


def test_adam_step_and_training(dataset):
    from oracle import prior_oracle as PO
    insts, _, pr, cnt, offs = dataset
    p0 = pr.params().astype(np.float64)
    all_ids = np.arange(cnt, dtype=np.int32)
    _, g = pr.gradient(all_ids)
    pr.set_params(p0.astype(np.float32))
    pr.train(1, batch=cnt, lr=1e-3, seed=5)  # one step over every example
    p1 = pr.params().astype(np.float64)
    exp, _, _ = PO.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g.astype(np.float64), 1, 1e-3)
    assert np.abs(p1 - exp).max() < 1e-5
    pr.set_params(p0.astype(np.float32))
    losses = pr.train(12, batch=256, lr=3e-3, seed=6)
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.8 * losses[0]
    # bit-reproducible: per-block partial gradients summed in a fixed order
    trained = pr.params()
    pr.set_params(p0.astype(np.float32))
    assert np.array_equal(pr.train(12, batch=256, lr=3e-3, seed=6), losses)
    assert np.array_equal(pr.params(), trained)
    l1, g1 = pr.gradient(all_ids[:100])
    l2, g2 = pr.gradient(all_ids[:100])
    assert l1 == l2 and np.array_equal(g1, g2)


def test_learned_levels_drive_the_exact_construct(dataset, native, oracle_mod):
    """Levels from the learned scores (oracle mapping of the device scores),
    and routes built on them bit-exact against the oracle construct."""
    from oracle import prior_oracle as PO
    insts, _, pr, _, offs = dataset
    inst, off = insts[2], int(offs[2])
    _, kv, sc = pr.rows(off, inst.n + 1, scores=True)
    with native.Context(0) as c:
        c.setup_instance(inst, ants=24, cand_k=K_CAND, seed=9)
        cand0, lvl0 = c.candidates()
        c.apply_prior(pr, 1.5)
        cand, lvl = c.candidates()
        assert np.array_equal(cand, cand0)
        exp = PO.levels(sc, kv, K_CAND, 1.5)
        assert np.array_equal(lvl.reshape(-1, K_CAND).astype(np.int64), exp)
        assert not np.array_equal(lvl, lvl0)
        A, lut, _ = oracle_mod.tables()
        tau = c.tau()
        w = oracle_mod.weights(inst.n, K_CAND, cand, lvl, tau, A, lut)
        assert np.array_equal(c.weights(), w)
        c.construct(0)
        nodes, lens, cost, feas, steps, draws = c.ants()
        for a in range(24):
            f, on, ol, oc, os_, od = oracle_mod.construct_ant(
                inst.x, inst.y, inst.demand, inst.vehicles, inst.capacity, K_CAND, cand, w,
                9, 0, a)
            assert bool(feas[a]) == f and np.array_equal(lens[a], ol)
            assert np.array_equal(nodes[a][: int(ol.sum())], on) and draws[a] == od
        c.apply_prior(None)
        assert np.array_equal(c.candidates()[1], lvl0)


def test_batch_levels_equal_context_levels(dataset, native):
    insts, _, pr, _, _ = dataset
    with native.Batch(0) as b:
        b.setup(insts, ants=32, cand_k=16, seed=77, epochs=12)
        b.apply_prior(pr, 1.0)
        b.solve()
        for i, inst in enumerate(insts):
            with native.Context(0) as c:
                c.setup_instance(inst, ants=32, cand_k=16, seed=77 + i, fixed_epochs=12)
                c.apply_prior(pr, 1.0)
                st = c.run(12)
                bn, bl, bc, be = b.best(i)
                nodes, lens, cost = c.best()
                assert bc == cost and np.array_equal(bn, nodes) and np.array_equal(bl, lens)


def test_cli_learned_prior_and_plain_fallback(dataset, tmp_path):
    import os
    import subprocess
    _, _, pr, _, _ = dataset
    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "aco_vrp_cuda.out")
    params = tmp_path / "prior.bin"
    pr.save(str(params))
    inst = I.uniform_instance(60, 3, 816)
    vrp = tmp_path / "i.vrp"
    I.write_vrp(inst, str(vrp))
    env = dict(os.environ, ACO_SOLVER_FIXED_EPOCHS="20", ACO_SOLVER_STAGNATION_EPOCHS="0",
               ACO_SOLVER_PROGRESS_INTERVAL_SECONDS="0", ACO_CUDA_PRIOR="learned",
               ACO_CUDA_PRIOR_FILE=str(params))
    r = subprocess.run([cli, str(vrp), "3", "32", "5"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "best cost:" in r.stdout, r.stderr
    assert "unavailable" not in r.stderr
    env["ACO_CUDA_PRIOR_FILE"] = str(tmp_path / "missing.bin")
    r2 = subprocess.run([cli, str(vrp), "3", "32", "5"], env=env, capture_output=True,
                        text=True, timeout=120)
    assert r2.returncode == 0 and "best cost:" in r2.stdout
    assert "learned prior unavailable" in r2.stderr
    env["ACO_CUDA_PRIOR"] = "plain"
    r3 = subprocess.run([cli, str(vrp), "3", "32", "5"], env=env, capture_output=True,
                        text=True, timeout=120)
    # a missing file falls back to exactly the plain solver
    assert r3.returncode == 0
    assert r3.stdout.split("best cost:")[1] == r2.stdout.split("best cost:")[1]


def test_time_to_cost_pipeline(dataset):
    from vehicleroutingproblem_b200 import prior as PR
    _, _, pr, _, _ = dataset
    res = PR.time_to_cost([I.uniform_instance(150, 3, 817)], pr, gamma=1.0, epochs=30,
                          ants=32, cand_k=32)
    row = res["rows"][0]
    assert res["instances"] == 1 and 1 <= row["plain_epochs"] <= 30
    assert row["plain_s"] > 0 and row["learned_s"] > 0 and row["prior_s"] > 0


def test_learned_prior_gains_over_plain_eta():
    """What the trained network gains over the method without it: on
    held-out n=1000 instances the learned levels reach the plain solver's
    final cost (+0.5 %, FP64) in under half its time.  The control -- the
    plain solver with a hand-tuned sharper eta^8 -- is reported, not
    asserted: it does about as well, since the network mostly learns a
    sharper preference for near candidates."""
    import json
    from vehicleroutingproblem_b200 import prior as PR
    tr = I.prior_training_instances(256)
    sols = PR.elite_solutions(tr, ants=64, cand_k=16, epochs=120)
    with _native.Prior(0, seed=1) as pr:
        count = pr.set_dataset(tr, [(x[0], x[1]) for x in sols], cand_k=32)
        losses = pr.train(10, batch=4096, lr=2e-3, seed=11)
        assert count > 0 and losses[-1] < losses[0]
        held = I.prior_heldout_instances(4)
        res = PR.time_to_cost(held, pr, gamma=4.0, epochs=300, ants=256, cand_k=32,
                              control_beta=8.0)
    print(json.dumps({"learned_vs_plain_time_ratio": res["time_ratio_of_sums"],
                      "control_beta8_vs_plain_time_ratio": res["control"]["time_ratio_of_sums"],
                      "learned_vs_control_final_cost": res["control"][
                          "learned_vs_control_final_cost_mean"]}))
    assert res["hit_rate"] == 1.0
    assert res["time_ratio_of_sums"] < 0.5


def test_residual_levels_add_to_plain(dataset, native):
    from oracle import prior_oracle as PO
    insts, _, pr, _, offs = dataset
    inst, off = insts[1], int(offs[1])
    _, kv, sc = pr.rows(off, inst.n + 1, scores=True)
    with native.Context(0) as c:
        c.setup_instance(inst, ants=16, cand_k=K_CAND, seed=3)
        _, plain = c.candidates()
        c.apply_prior(pr, 2.0, residual=True)
        _, lvl = c.candidates()
        learned = PO.levels(sc, kv, K_CAND, 2.0)
        plain = plain.reshape(-1, K_CAND).astype(np.int64)
        valid = np.arange(K_CAND)[None, :] < kv[:, None]
        exp = np.where(valid, np.minimum(4095, plain + learned), 4095)
        assert np.array_equal(lvl.reshape(-1, K_CAND).astype(np.int64), exp)
        c.apply_prior(pr, 2.0, residual=True)  # applying again starts from the plain levels
        assert np.array_equal(c.candidates()[1], lvl)
