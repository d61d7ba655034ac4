"""The sequential path's FP64 pheromone update on the GPU
(aco_b200_seq_pheromone_update, src/seq/aco_sequential.c:829-886) against
the oracle's restatement, bit for bit, through the C ABI: evaporation, the
iteration-best and global-best deposits, the MMAS clamp and the stagnation
reset, with and without a global best, on solutions that include empty
routes, for two calls in a row on one scratch bitmap."""
import numpy as np
import pytest

from vehicleroutingproblem_b200 import _native
from vehicleroutingproblem_b200 import instances as I

pytestmark = pytest.mark.gpu


def _solutions(inst, k, ants, seed):
    with _native.Context(0) as ctx:
        ctx.setup_instance(inst, ants=ants, cand_k=k, seed=seed)
        ctx.construct(1)
        nodes, lens, cost, feas, _, _ = ctx.ants()
    sols = []
    for a in (0, 1):
        ln = lens[a]
        sols.append((nodes[a][: ln.sum()].astype(np.int32), ln.astype(np.int32), float(cost[a])))
    return sols


def _many():
    b = I.uniform_instance(300, 60, 972).unit_twin()
    return b.x, b.y, b.demand


# (n+1)^2 is odd for even n (the last cell, on the diagonal, is left out of
# the 16-byte pairs) and even for odd n: both are covered.
CASES = [("u50", lambda: I.uniform_instance(50, 3, 971), 16),
         ("u301", lambda: I.uniform_instance(301, 4, 974), 16),
         ("u300_empty_routes", lambda: I.Instance("er", *_many(), 60, 8), 16),
         ("n1000", I.workload_n1000, 32),
         ("u3000", lambda: I.uniform_instance(3000, 12, 973), 32)]


@pytest.mark.parametrize("name,factory,k", CASES)
@pytest.mark.parametrize("reset,with_global", [(False, True), (True, True), (False, False)])
def test_seq_update_matches_oracle(oracle_mod, name, factory, k, reset, with_global):
    import torch
    L = _native.load()
    inst = factory()
    n, K = inst.n, inst.vehicles
    (itn, itl, itc), (gbn, gbl, gbc) = _solutions(inst, k, 4, 31)
    rho, tau0 = 0.1, 1.0
    tau_max = 1.0 / ((1.0 - rho) * gbc)
    tau_min = tau_max * 0.05
    rs = np.random.RandomState(n + 7 * reset)
    tau = rs.uniform(0.5 * tau_min, 2.0 * tau_max, size=(n + 1) ** 2)
    d_it = 0.3 * 1.0 / itc
    d_gb = 0.7 * 1.0 / gbc
    d_tau = torch.from_numpy(tau.copy()).cuda()
    d_in, d_il = torch.from_numpy(itn).cuda(), torch.from_numpy(itl).cuda()
    d_gn, d_gl = torch.from_numpy(gbn).cuda(), torch.from_numpy(gbl).cuda()
    scratch = torch.zeros(L.aco_b200_seq_update_scratch_bytes(n), dtype=torch.uint8,
                          device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    expected = tau
    for call in range(2):
        expected = oracle_mod.seq_pheromone_update(
            expected, n, itn, itl, d_it, gbn if with_global else None, gbl, d_gb, rho,
            tau_min, tau_max, reset, tau0)
        rc = L.aco_b200_seq_pheromone_update(
            d_tau.data_ptr(), n, K, d_in.data_ptr(), d_il.data_ptr(), d_it,
            d_gn.data_ptr() if with_global else None, d_gl.data_ptr() if with_global else None,
            d_gb, rho, tau_min, tau_max, 1 if reset else 0, tau0, scratch.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = d_tau.cpu().numpy()
        assert np.array_equal(got.view(np.uint64), expected.view(np.uint64)), f"call {call + 1}"
        assert int(scratch.sum()) == 0  # the bitmap is left zeroed


def test_seq_update_rejects_bad_arguments():
    import torch
    L = _native.load()
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    ib = torch.zeros(16, dtype=torch.int32, device="cuda")
    args = [buf.data_ptr(), 5, 2, ib.data_ptr(), ib.data_ptr(), 1.0, None, None, 0.0, 0.1,
            0.1, 1.0, 0, 1.0, buf.data_ptr(), None]
    bad_k = list(args)
    bad_k[2] = 9000  # more routes than the kernels stage
    assert L.aco_b200_seq_pheromone_update(*bad_k) == _native.ACO_ERR_INVALID_INPUT
    bad_clamp = list(args)
    bad_clamp[10], bad_clamp[11] = 2.0, 1.0  # tau_min > tau_max
    assert L.aco_b200_seq_pheromone_update(*bad_clamp) == _native.ACO_ERR_INVALID_INPUT
    half = list(args)
    half[6] = ib.data_ptr()  # best nodes without best lengths
    assert L.aco_b200_seq_pheromone_update(*half) == _native.ACO_ERR_INVALID_INPUT
    odd = list(args)
    odd[0] = buf.data_ptr() + 8  # not 16-byte aligned
    assert L.aco_b200_seq_pheromone_update(*odd) == _native.ACO_ERR_INVALID_INPUT
