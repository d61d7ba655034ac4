"""CPU checks of the prior's FP64 oracle: its backward pass against central
finite differences of its loss, BF16 rounding, features, levels."""
import numpy as np

from oracle import prior_oracle as PO
from vehicleroutingproblem_b200 import instances as I


def test_backward_matches_finite_differences():
    rs = np.random.RandomState(0)
    X = rs.rand(6, 32, 8)
    kv = np.array([32, 20, 5, 32, 1, 12])
    ex = np.array([[0, 3], [1, 19], [2, 0], [3, 31], [5, 7], [0, 1]])
    p = rs.randn(PO.N_PARAMS) * 0.3
    _, g = PO.loss_grad(p, X, kv, ex, mimic=False)
    idx = np.concatenate([rs.choice(PO.N_PARAMS, 60, replace=False),
                          [PO.P_B3, PO.P_B1 + 3, PO.P_B2 + 5, PO.P_W3 + 2, PO.P_W1 + 9]])
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp = PO.loss_only(q, X, kv, ex)
        q[i] -= 2 * eps
        lm = PO.loss_only(q, X, kv, ex)
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-7 + 1e-5 * abs(g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, 3.14159, -2.5e-3, 0.0, 65504.0])
    r = PO.bf16(v)
    assert list(r[:4]) == [1.0, 1.0, 1.0078125, 3.140625]  # ties to even, nearest
    bits = (np.asarray(r, np.float32).view(np.uint32) >> 16).astype(np.uint16)
    assert np.array_equal(PO.bf16_bits_to_float(bits), r)


def test_features_shape_and_ranges(oracle_mod):
    inst = I.uniform_instance(60, 3, 17)
    k = 32
    cand = oracle_mod.knn(inst.x, inst.y, k)
    F, kv = PO.features(inst.x, inst.y, inst.demand, inst.capacity, cand, k)
    assert F.shape == (61, 32, 8) and np.all(kv == 32)
    assert np.all(F[..., 0] <= 1) and np.all(F[:, 0, 1] == 1)  # nearest slot: ratio 1
    assert np.all(F[0, :, 6] == 0)  # depot row: no angle
    assert set(np.unique(F[..., 7])) <= {0.0, 1.0}


def test_levels_mapping():
    sc = np.zeros((2, 32), np.float32)
    sc[0, :3] = [2.0, 1.0, -1.0]
    kv = np.array([3, 0])
    L = PO.levels(sc, kv, 4, 1.0)
    step = 16 / np.log(2)
    assert list(L[0]) == [0, int(np.rint(step)), int(np.rint(3 * step)), 4095]
    assert list(L[1]) == [4095] * 4
